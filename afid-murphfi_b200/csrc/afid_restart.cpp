// afid_restart.cpp — ReadFlowInterp as a whole (include/afid_continua.h): the same-grid restart,
// or, when the continua files come from another grid, the interpolating restart of
// ReadFlowInterp.F90:85-136:
//   CreateOldGrid          multires/IC_interpolation/CreateOldGrid.F90:11-115
//   CreateInputStencil     CreateNewInputStencil.F90:1-41 (only the cell-centre stencils are used)
//   InterpInputVel         InterpInputVel.F90:1-350
//   CreateSalStencil +     CreateNewSalStencil.F90, InterpInputSal.F90 (refined salinity)
//   InterpInputSal
// Interpolation is the tensor-product Hermite form of interpolate_xyz_old_to_new
// (HermiteInterpolations.F90:314-346), evaluated per new point from per-target stencil tables and
// contracted in the reference's order (z, then y, then x).  Velocities are rebuilt from their
// interpolated gradients: vx integrated from vx(1) = 0 along x, vy from an interpolated y = 0 plane
// along y, vz from an interpolated z = 0 plane along z.  One rank: the MPI_SCAN offsets vanish.
// This runs once per restart on the host, as it does in the reference.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "afid_continua.h"
#include "afid_host_internal.h"
#include "afid_salinity.h"

namespace {

struct Axis {
  std::vector<int> start;  // first source row of each new point (0-based; x: row -1 is -1)
  std::vector<double> w;   // 4 weights per new point
};

// Centre-to-centre stencil old -> new along one axis (interval loops io = 0 .. n_old).
bool make_axis(const std::vector<double> &xo, const std::vector<double> &xn, double len, char axis, Axis &a) {
  const std::vector<int> idx = afid_hostd::interpolation_indices(xo, xn, len);
  a.w = afid_hostd::construct_stencil(xo, xn, len, idx, axis);
  return afid_hostd::starts_from_intervals(idx, (int)xn.size(), 0, (int)xo.size(), a.start);
}

std::vector<double> centres(const std::vector<double> &c) {
  std::vector<double> m(c.size() - 1);
  for (size_t k = 0; k + 1 < c.size(); ++k) m[k] = (c[k] + c[k + 1]) * 0.5;
  return m;
}

// An x-extended old field: Fortran rows -1 .. n+2 at 0 .. n+3 (row 0 and row n+1 are the wall
// ghosts, rows -1 and n+2 zero), y/z periodic.
struct Ext {
  int nz, ny, n;  // old sizes; rows per column n + 4
  std::vector<double> v;
  Ext(int nz_, int ny_, int n_) : nz(nz_), ny(ny_), n(n_), v((size_t)nz_ * ny_ * (n_ + 4), 0.0) {}
  double *col(int i, int j) { return &v[((size_t)i * ny + j) * (n + 4)]; }
};

// out[(i * ny_new + j) * ldo + k] = sum_c wz_c sum_b wy_b sum_a wx_a e(z_c, y_b, x_a), for the
// new points k < nx_new, j < ny_new, i < nz_new.
void interp3(Ext &e, const Axis &ax, const Axis &ay, const Axis &az, double *out, int ldo) {
  const int nxn = (int)ax.start.size(), nyn = (int)ay.start.size(), nzn = (int)az.start.size();
  const int rows = e.n + 4;
  std::vector<double> q2((size_t)e.ny * rows), q1(rows);
  for (int icr = 0; icr < nzn; ++icr) {
    int zi[4];
    for (int c = 0; c < 4; ++c) zi[c] = ((az.start[icr] + c) % e.nz + e.nz) % e.nz;
    const double *wz = &az.w[4 * (size_t)icr];
    for (int j = 0; j < e.ny; ++j) {
      double *q = &q2[(size_t)j * rows];
      const double *s0 = e.col(zi[0], j), *s1 = e.col(zi[1], j), *s2 = e.col(zi[2], j), *s3 = e.col(zi[3], j);
      for (int r = 0; r < rows; ++r) q[r] = s0[r] * wz[0] + s1[r] * wz[1] + s2[r] * wz[2] + s3[r] * wz[3];
    }
    for (int jcr = 0; jcr < nyn; ++jcr) {
      int yj[4];
      for (int b = 0; b < 4; ++b) yj[b] = ((ay.start[jcr] + b) % e.ny + e.ny) % e.ny;
      const double *wy = &ay.w[4 * (size_t)jcr];
      const double *r0 = &q2[(size_t)yj[0] * rows], *r1 = &q2[(size_t)yj[1] * rows], *r2 = &q2[(size_t)yj[2] * rows],
                   *r3 = &q2[(size_t)yj[3] * rows];
      for (int r = 0; r < rows; ++r) q1[r] = r0[r] * wy[0] + r1[r] * wy[1] + r2[r] * wy[2] + r3[r] * wy[3];
      double *o = out + ((size_t)icr * nyn + jcr) * ldo;
      for (int kcr = 0; kcr < nxn; ++kcr) {
        const double *wx = &ax.w[4 * (size_t)kcr];
        const double *x = &q1[(size_t)ax.start[kcr] + 2];
        o[kcr] = x[0] * wx[0] + x[1] * wx[1] + x[2] * wx[2] + x[3] * wx[3];
      }
    }
  }
}

// The first-guess plane: plane[p * (n + 4) + r] with one periodic axis (extent np) and x rows
// -1 .. n+2; contracted along the periodic axis first, then x.  New point pc of the periodic axis
// goes to out + pc * stride_p.
void interp2(const std::vector<double> &plane, int np, int n, const Axis &ax, const Axis &ap, double *out,
             size_t stride_p) {
  const int rows = n + 4, nxn = (int)ax.start.size(), npn = (int)ap.start.size();
  std::vector<double> q1(rows);
  for (int pc = 0; pc < npn; ++pc) {
    int pi[4];
    for (int b = 0; b < 4; ++b) pi[b] = ((ap.start[pc] + b) % np + np) % np;
    const double *w = &ap.w[4 * (size_t)pc];
    for (int r = 0; r < rows; ++r)
      q1[r] = plane[(size_t)pi[0] * rows + r] * w[0] + plane[(size_t)pi[1] * rows + r] * w[1] +
              plane[(size_t)pi[2] * rows + r] * w[2] + plane[(size_t)pi[3] * rows + r] * w[3];
    double *o = out + (size_t)pc * stride_p;
    for (int kcr = 0; kcr < nxn; ++kcr) {
      const double *wx = &ax.w[4 * (size_t)kcr];
      const double *x = &q1[(size_t)ax.start[kcr] + 2];
      o[kcr] = x[0] * wx[0] + x[1] * wx[1] + x[2] * wx[2] + x[3] * wx[3];
    }
  }
}

int read_var(const std::string &path, std::vector<double> &v, int n1, int n2, int n3) {
  int dtype = 0, rank = 0;
  int64_t dims[AFID_H5_MAX_RANK];
  int s = afid_h5_info(path.c_str(), "var", &dtype, &rank, dims);
  if (s != AFID_OK) return s;
  if (rank != 3 || dims[0] != n3 || dims[1] != n2 || dims[2] != n1) return AFID_E_INVALID;
  v.resize((size_t)n1 * n2 * n3);
  return afid_h5_read_f64(path.c_str(), "var", v.data(), (int64_t)v.size());
}

}  // namespace

extern "C" int afid_read_flow_interp(const char *dir, const afid_input_t *in, double *time_out, double *vx,
                                     double *vy, double *vz, double *temp, double *pr, int *pr_read,
                                     int *interpolated, double *sal) {
  return afid_guard([&]() -> int {
    if (!dir || !in || !vx || !vy || !vz || !temp) return AFID_E_INVALID;
    afid_continua_master_t cur{};
    int s = afid_continua_master_from_input(in, 0.0, &cur);
    if (s != AFID_OK) return s;
    const bool want_sal = in->multires && sal;
    cur.multires = in->multires ? 1 : 0;
    afid_continua_master_t old{};
    if ((s = afid_read_continua_master(dir, cur.multires, &old)) != AFID_OK) return s;
    if (std::fabs(cur.ylen - old.ylen) > 1e-8 || std::fabs(cur.zlen - old.zlen) > 1e-8) return AFID_E_INVALID;
    const bool same = cur.nx == old.nx && cur.ny == old.ny && cur.nz == old.nz && cur.istr3 == old.istr3 &&
                      std::fabs(cur.str3 - old.str3) <= 1e-8 &&
                      (!cur.multires || (cur.nxr == old.nxr && cur.nyr == old.nyr && cur.nzr == old.nzr &&
                                         cur.istr3r == old.istr3r));
    if (interpolated) *interpolated = same ? 0 : 1;
    if (same)
      return afid_read_flow_field(dir, &cur, time_out, vx, vy, vz, temp, pr, pr_read, want_sal ? sal : nullptr);

    // ---- CreateOldGrid / current grid ----
    const int nxo = old.nx, nxmo = nxo - 1, nymo = old.ny - 1, nzmo = old.nz - 1;
    if (nxmo < 2 || nymo < 1 || nzmo < 1 || (nzmo == 1) != (in->nzm == 1)) return AFID_E_INVALID;
    const double pi = 2.0 * std::asin(1.0);
    std::vector<double> xco, yco, ymo, zco, zmo, xc, yc, ym, zc, zm;
    if (afid_hostd::x_grid(old.istr3, nxmo, in->alx3, old.str3, pi, 1.0, xco) != AFID_OK) return AFID_E_INVALID;
    afid_hostd::uniform_grid(yco, ymo, nymo, in->ylen);
    afid_hostd::uniform_grid(zco, zmo, nzmo, in->zlen);
    const int nxm = in->nxm, nym = in->nym, nzm = in->nzm, nx = nxm + 1;
    if (afid_hostd::x_grid(in->istr3, nxm, in->alx3, in->str3, pi, 1.0, xc) != AFID_OK) return AFID_E_INVALID;
    afid_hostd::uniform_grid(yc, ym, nym, in->ylen);
    afid_hostd::uniform_grid(zc, zm, nzm, in->zlen);
    const std::vector<double> xmo = centres(xco), xm = centres(xc);
    Axis ax, ay, az;  // CreateInputStencil: cell centres to cell centres
    if (!make_axis(xmo, xm, in->alx3, 'x', ax) || !make_axis(ymo, ym, in->ylen, 'y', ay) ||
        !make_axis(zmo, zm, in->zlen, 'z', az))
      return AFID_E_INVALID;

    const std::string base = std::string(dir) + "/continua";
    std::vector<double> f;
    const size_t plane = (size_t)nym * nx, ncell = plane * nzm;
    std::fill(vx, vx + ncell, 0.0);
    std::fill(vy, vy + ncell, 0.0);
    std::fill(vz, vz + ncell, 0.0);
    std::fill(temp, temp + ncell, 0.0);
    std::vector<double> grad(ncell);  // tpdv on the new grid, x stride nx
    Ext e(nzmo, nymo, nxmo);
    auto wall_rows = [&](Ext &x) {  // rows 0 and nxo: (1 - 2 inslw) * rows 1 and nxmo
      for (int i = 0; i < nzmo; ++i)
        for (int j = 0; j < nymo; ++j) {
          double *c = x.col(i, j);
          c[1] = (1 - 2 * in->inslws) * c[2];
          c[nxmo + 2] = (1 - 2 * in->inslwn) * c[nxmo + 1];
        }
    };
    // ---- vx: dvx/dx at the old centres, interpolated, integrated from vx(1) = 0 ----
    if ((s = read_var(base + "_vx.h5", f, nxo, nymo, nzmo)) != AFID_OK) return s;
    for (int i = 0; i < nzmo; ++i)
      for (int j = 0; j < nymo; ++j) {
        const double *v = &f[((size_t)i * nymo + j) * nxo];
        double *c = e.col(i, j);
        for (int k = 0; k < nxmo; ++k) c[k + 2] = (v[k + 1] - v[k]) / (xco[k + 1] - xco[k]);
      }
    wall_rows(e);
    interp3(e, ax, ay, az, grad.data(), nx);
    for (size_t c = 0; c < (size_t)nym * nzm; ++c) {
      double *v = vx + c * nx;
      const double *g = &grad[c * nx];
      v[0] = 0.0;
      for (int k = 0; k < nxm; ++k) v[k + 1] = v[k] + g[k] * (xc[k + 1] - xc[k]);
    }
    // ---- vy: dvy/dy, the y = 0 plane interpolated in x-z, integrated along y ----
    if ((s = read_var(base + "_vy.h5", f, nxo, nymo, nzmo)) != AFID_OK) return s;
    const double dyo = 1.0 / (yco[1] - yco[0]), dzo = 1.0 / (zco[1] - zco[0]);
    for (int i = 0; i < nzmo; ++i)
      for (int j = 0; j < nymo; ++j) {
        const double *v = &f[((size_t)i * nymo + j) * nxo], *vp = &f[((size_t)i * nymo + (j + 1) % nymo) * nxo];
        double *c = e.col(i, j);
        for (int k = 0; k < nxmo; ++k) c[k + 2] = (vp[k] - v[k]) * dyo;
      }
    wall_rows(e);
    interp3(e, ax, ay, az, grad.data(), nx);
    {
      std::vector<double> pl((size_t)nzmo * (nxmo + 4), 0.0);
      for (int i = 0; i < nzmo; ++i) {
        const double *v = &f[((size_t)i * nymo) * nxo];
        double *c = &pl[(size_t)i * (nxmo + 4)];
        for (int k = 0; k < nxmo; ++k) c[k + 2] = v[k];
        c[1] = (1 - 2 * in->inslws) * c[2];
        c[nxmo + 2] = (1 - 2 * in->inslwn) * c[nxmo + 1];
      }
      interp2(pl, nzmo, nxmo, ax, az, vy, plane);  // vy(:, 1, :) of every new z plane
    }
    const double lya = 1.0 / ((double)nym / in->ylen), lza = 1.0 / ((double)nzm / in->zlen);
    for (int i = 0; i < nzm; ++i)
      for (int j = 0; j + 1 < nym; ++j) {
        double *v = vy + (size_t)i * plane + (size_t)j * nx;
        const double *g = &grad[(size_t)i * plane + (size_t)j * nx];
        for (int k = 0; k < nxm; ++k) v[nx + k] = v[k] + g[k] * lya;
      }
    // ---- vz: dvz/dz, the z = 0 plane interpolated in x-y, integrated along z ----
    if ((s = read_var(base + "_vz.h5", f, nxo, nymo, nzmo)) != AFID_OK) return s;
    for (int i = 0; i < nzmo; ++i)
      for (int j = 0; j < nymo; ++j) {
        const double *v = &f[((size_t)i * nymo + j) * nxo], *vp = &f[((size_t)((i + 1) % nzmo) * nymo + j) * nxo];
        double *c = e.col(i, j);
        for (int k = 0; k < nxmo; ++k) c[k + 2] = (vp[k] - v[k]) * dzo;
      }
    wall_rows(e);
    interp3(e, ax, ay, az, grad.data(), nx);
    {
      std::vector<double> pl((size_t)nymo * (nxmo + 4), 0.0);
      for (int j = 0; j < nymo; ++j) {
        const double *v = &f[(size_t)j * nxo];
        double *c = &pl[(size_t)j * (nxmo + 4)];
        for (int k = 0; k < nxmo; ++k) c[k + 2] = v[k];
        c[1] = (1 - 2 * in->inslws) * c[2];
        c[nxmo + 2] = (1 - 2 * in->inslwn) * c[nxmo + 1];
      }
      interp2(pl, nymo, nxmo, ax, ay, vz, nx);  // vz(:, :, 1)
    }
    for (int i = 0; i + 1 < nzm; ++i)
      for (int j = 0; j < nym; ++j) {
        double *v = vz + (size_t)i * plane + (size_t)j * nx;
        const double *g = &grad[(size_t)i * plane + (size_t)j * nx];
        for (int k = 0; k < nxm; ++k) v[plane + k] = v[k] + g[k] * lza;
      }
    // ---- temperature with the plate ghosts ----
    if ((s = read_var(base + "_temp.h5", f, nxo, nymo, nzmo)) != AFID_OK) return s;
    double tlo, tup;
    if (in->rayt > 0) {
      tup = in->inslwn == 0 ? 0.0 : -0.5;
      tlo = in->inslwn == 0 ? 1.0 : 0.5;
    } else {
      tup = 0.5;
      tlo = -0.5;
    }
    for (int i = 0; i < nzmo; ++i)
      for (int j = 0; j < nymo; ++j) {
        const double *v = &f[((size_t)i * nymo + j) * nxo];
        double *c = e.col(i, j);
        for (int k = 0; k < nxmo; ++k) c[k + 2] = v[k];
        c[1] = in->tfixs == 1 ? 2.0 * tlo - v[0] : v[0];
        c[nxmo + 2] = in->tfixn == 1 ? 2.0 * tup - v[nxmo - 1] : v[nxmo - 1];
      }
    interp3(e, ax, ay, az, temp, nx);
    for (size_t c = 0; c < (size_t)nym * nzm; ++c) temp[c * nx + nxm] = 0.0;
    // ---- refined salinity ----
    if (want_sal) {
      const int nxmro = old.nxr - 1, nymro = old.nyr - 1, nzmro = old.nzr - 1;
      const int nxmr = in->nxmr, nymr = in->nymr, nzmr = in->nzmr;
      if (nxmro < 2 || nymro < 1 || nzmro < 1) return AFID_E_INVALID;
      std::vector<double> xcro, ycro, ymro, zcro, zmro, xcr, ycr, ymr, zcr, zmr;
      // CreateOldGrid.F90: the old refined grid takes the old STR3 and Schmidt number 1
      if (afid_hostd::x_grid(old.istr3r, nxmro, in->alx3, old.str3, pi, 1.0, xcro) != AFID_OK) return AFID_E_INVALID;
      afid_hostd::uniform_grid(ycro, ymro, nymro, in->ylen);
      afid_hostd::uniform_grid(zcro, zmro, nzmro, in->zlen);
      // CreateMgrdGrid.F90: the current refined grid (as afid_mgrd_create builds it)
      if (afid_hostd::x_grid(in->istr3r, nxmr, in->alx3, in->str3, pi, in->pras, xcr) != AFID_OK) return AFID_E_INVALID;
      afid_hostd::uniform_grid(ycr, ymr, nymr, in->ylen);
      afid_hostd::uniform_grid(zcr, zmr, nzmr, in->zlen);
      Axis rx, ry, rz;
      if (!make_axis(centres(xcro), centres(xcr), in->alx3, 'x', rx) || !make_axis(ymro, ymr, in->ylen, 'y', ry) ||
          !make_axis(zmro, zmr, in->zlen, 'z', rz))
        return AFID_E_INVALID;
      if ((s = read_var(base + "_sal.h5", f, nxmro + 1, nymro, nzmro)) != AFID_OK) return s;
      const double slo = in->rays > 0 ? -0.5 : 0.5, sup = in->rays > 0 ? 0.5 : -0.5;
      Ext es(nzmro, nymro, nxmro);
      for (int i = 0; i < nzmro; ++i)
        for (int j = 0; j < nymro; ++j) {
          const double *v = &f[((size_t)i * nymro + j) * (nxmro + 1)];
          double *c = es.col(i, j);
          for (int k = 0; k < nxmro; ++k) c[k + 2] = v[k];
          c[1] = in->sfixs == 1 ? 2.0 * slo - v[0] : v[0];
          c[nxmro + 2] = in->sfixn == 1 ? 2.0 * sup - v[nxmro - 1] : v[nxmro - 1];
        }
      interp3(es, rx, ry, rz, sal, nxmr);
    }
    // the pressure is not read in this branch (it stays zero)
    if (pr) std::fill(pr, pr + ncell, 0.0);
    if (pr_read) *pr_read = 0;
    if (time_out) *time_out = old.time;
    return AFID_OK;
  });
}

extern "C" int afid_gpu_read_flow_interp(afid_ctx_t *ctx, const char *dir, const afid_input_t *in, double *time_out,
                                         int *interpolated) {
  return afid_guard([&]() -> int {
    if (!ctx || !dir || !in) return AFID_E_INVALID;
    int dims[6];
    int s = afid_gpu_dims(ctx, dims);
    if (s != AFID_OK) return s;
    if (in->nxm != dims[0] || in->nym != dims[1] || in->nzm != dims[2]) return AFID_E_INVALID;
    const bool with_sal = in->multires && dims[3] > 0;
    if (with_sal && (in->nxmr != dims[3] || in->nymr != dims[4] || in->nzmr != dims[5])) return AFID_E_INVALID;
    const int nx = dims[0] + 1, nym = dims[1], nzm = dims[2];
    const size_t n = (size_t)nx * nym * nzm;
    std::vector<double> fl(5 * n, 0.0);
    double *vx = fl.data(), *vy = vx + n, *vz = vy + n, *temp = vz + n, *pr = temp + n;
    std::vector<double> sal(with_sal ? (size_t)dims[3] * dims[4] * dims[5] : 0);
    int pr_read = 0, interp = 0;
    double t = 0.0;
    if ((s = afid_read_flow_interp(dir, in, &t, vx, vy, vz, temp, pr, &pr_read, &interp,
                                   with_sal ? sal.data() : nullptr)) != AFID_OK)
      return s;
    if ((s = afid_gpu_upload(ctx, vx, vy, vz, temp, pr, nx, nym)) != AFID_OK) return s;
    if (with_sal && (s = afid_gpu_sal_upload(ctx, sal.data(), dims[3], dims[4])) != AFID_OK) return s;
    if (time_out) *time_out = t;
    if (interpolated) *interpolated = interp;
    return AFID_OK;
  });
}
