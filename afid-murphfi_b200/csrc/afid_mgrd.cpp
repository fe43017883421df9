// afid_mgrd.cpp — host set-up of the refined salinity grid (include/afid_salinity.h):
// CreateMgrdGrid.F90 (refined metrics), CreateMgrdStencil.F90 with the Hermite stencils of
// multires/HermiteInterpolations.F90:26-164, SetSalBCs and CreateInitialSalinity.
//
// The reference keeps its stencils as Fortran index arrays (irangs, ...) plus weights that its
// interpolation loops walk interval by interval.  Here every stencil is turned into a per-target
// table (first source row + 4 weights) that a GPU thread can evaluate on its own.
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <new>

#include "afid_host_internal.h"
#include "afid_salinity.h"

using afid_hostd::philox_u;

namespace afid_hostd {

// HermiteInterpolations.F90:26-57: idx[io], io = 0 .. n_old+1 (Fortran values, 1-based), the
// first new index whose coordinate is >= x_old(io).
std::vector<int> interpolation_indices(const std::vector<double> &x_old, const std::vector<double> &x_new,
                                       double x_len) {
  const int n_old = (int)x_old.size(), n_new = (int)x_new.size();
  std::vector<double> xn(n_new + 2, 0.0);
  for (int i = 0; i < n_new; ++i) xn[i + 1] = x_new[i];
  xn[0] = -xn[1];
  if (xn[0] == xn[1] && n_new > 1) xn[0] = -xn[2];
  xn[n_new + 1] = 2.0 * x_len - xn[n_new];
  if (xn[n_new + 1] == xn[n_new] && n_new > 1) xn[n_new + 1] = 2.0 * x_len - xn[n_new - 1];
  std::vector<int> idx(n_old + 2, 0);
  idx[0] = 1;
  for (int io = 1; io <= n_old; ++io) {
    const double xo = x_old[io - 1];
    for (int in = 0; in <= n_new; ++in)
      if (xn[in] < xo && xn[in + 1] >= xo) idx[io] = in + 1;
  }
  idx[n_old + 1] = n_new + 1;
  return idx;
}

// HermiteInterpolations.F90:59-103: x_ext(i), i = 1-n_ext .. n_og+n_ext, mirrored over the
// walls.  Mirror points past the original grid (only for n_og <= n_ext, where the reference
// reads out of bounds) take the nearest point that exists; they only meet zero weights.
struct Ext {
  std::vector<double> v;
  int off;
  double operator()(int i) const { return v[(size_t)(i + off)]; }
};
Ext extend_grid(const std::vector<double> &x, double x_len, int n_ext) {
  const int n = (int)x.size();
  auto og = [&](int i) { return x[(size_t)(std::min(std::max(i, 1), n) - 1)]; };
  Ext e;
  e.off = n_ext - 1;
  e.v.assign(n + 2 * n_ext, 0.0);
  for (int i = 1; i <= n; ++i) e.v[i + e.off] = x[i - 1];
  const bool low_wall = std::fabs(x[0]) < 1e-10, up_wall = std::fabs(x[n - 1] - x_len) < 1e-10;
  for (int i = 1; i <= n_ext; ++i) {
    e.v[1 - i + e.off] = low_wall ? -og(1 + i) : -og(i);
    e.v[n + i + e.off] = up_wall ? 2 * x_len - og(n - i) : 2 * x_len - og(n + 1 - i);
  }
  return e;
}

// HermiteInterpolations.F90:105-164: weights cx[4*(in-1) + a] of every new point.
std::vector<double> construct_stencil(const std::vector<double> &x_old, const std::vector<double> &x_new,
                                      double x_len, const std::vector<int> &idx, char axis) {
  const int n_old = (int)x_old.size(), n_new = (int)x_new.size();
  std::vector<double> cx((size_t)4 * n_new, 0.0);
  const int n_ext = axis == 'x' ? 1 : 2;
  const Ext xo = extend_grid(x_old, x_len, n_ext), xn = extend_grid(x_new, x_len, n_ext);
  for (int io = 0; io <= n_old; ++io) {
    const int lo = std::max(idx[io], 1), hi = std::min(idx[io + 1] - 1, n_new);
    double *c;
    if (axis == 'x' && (io == 0 || io == n_old)) {
      const double dlc = xo(io + 1) - xo(io);
      for (int in = lo; in <= hi; ++in) {
        const double t = (xn(in) - xo(io)) / dlc;
        c = &cx[(size_t)4 * (in - 1)];
        c[0] = 0.0;
        c[1] = 1 - t;
        c[2] = t;
        c[3] = 0.0;
      }
    } else {
      const double dlm = xo(io) - xo(io - 1), dlc = xo(io + 1) - xo(io), dlp = xo(io + 2) - xo(io + 1);
      for (int in = lo; in <= hi; ++in) {
        const double t = (xn(in) - xo(io)) / dlc;
        c = &cx[(size_t)4 * (in - 1)];
        if (t < 1e-12) {
          c[0] = 0.0;
          c[1] = 1.0;
          c[2] = 0.0;
          c[3] = 0.0;
        } else {
          const double h00 = (1.0 + 2.0 * t) * (1.0 - t) * (1.0 - t);
          const double h10 = t * (1.0 - t) * (1.0 - t);
          const double h01 = (1.0 + 2.0 * (1.0 - t)) * t * t;
          const double h11 = -(1.0 - t) * t * t;
          c[0] = -h10 * dlc * dlc / dlm / (dlc + dlm);
          c[1] = h00 - h11 * dlp / (dlp + dlc) + h10 * (dlc - dlm) / dlm;
          c[2] = h01 + h10 * dlm / (dlm + dlc) + h11 * (dlp - dlc) / dlp;
          c[3] = h11 * dlc * dlc / dlp / (dlp + dlc);
        }
      }
    }
  }
  return cx;
}

// Per-target form of `do io = lo, hi; do in = max(idx(io),1), min(idx(io+1)-1, n_new)` whose body
// reads source rows io-1 .. io+2: the 0-based first source row of every new point.  False if a
// point is covered twice or not at all.
bool starts_from_intervals(const std::vector<int> &idx, int n_new, int io_lo, int io_hi, std::vector<int> &start) {
  const int unset = std::numeric_limits<int>::min();
  start.assign(n_new, unset);
  for (int io = io_lo; io <= io_hi; ++io)
    for (int in = std::max(idx[io], 1); in <= std::min(idx[io + 1] - 1, n_new); ++in) {
      if (start[in - 1] != unset) return false;
      start[in - 1] = io - 2;
    }
  for (int v : start)
    if (v == unset) return false;
  return true;
}

}  // namespace afid_hostd

using afid_hostd::construct_stencil;
using afid_hostd::interpolation_indices;
using afid_hostd::starts_from_intervals;

struct afid_mgrd {
  afid_sal_grid_t view{};
  int fast = 0;
  std::map<std::string, std::vector<double>> arr;
  std::vector<int> start[6];
  std::vector<double> w[6];
  std::vector<double> salbp, saltp;
  double salbp0 = -0.5, saltp0 = 0.5;
  int active_t = 1, gaxis = 1;
};

extern "C" {

static int mgrd_create(const afid_tables_t *coarse, afid_mgrd_t **out);

int afid_mgrd_create(const afid_tables_t *coarse, afid_mgrd_t **out) {
  if (!coarse || !out) return AFID_E_INVALID;
  *out = nullptr;
  try {
    return mgrd_create(coarse, out);
  } catch (const std::bad_alloc &) {
    return AFID_E_ALLOC;
  }
}

static int mgrd_create(const afid_tables_t *coarse, afid_mgrd_t **out) {
  const afid_input_t &in = coarse->in;
  const int nxm = in.nxm, nym = in.nym, nzm = in.nzm;
  const int nxmr = in.nxmr, nymr = in.nymr, nzmr = in.nzmr;
  if (!in.multires || !in.flagsal || in.flagpf || in.melt) return AFID_E_INVALID;
  if (nxmr < 3 || nymr < 1 || nzmr < 1 || nxmr > 1024 || nymr > (1 << 20) || nzmr > (1 << 20) ||
      (long long)nymr * nzmr > (1LL << 28))
    return AFID_E_INVALID;
  if ((nzm == 1) != (nzmr == 1)) return AFID_E_INVALID;
  if (in.gaxis < 1 || in.gaxis > 3) return AFID_E_INVALID;
  std::unique_ptr<afid_mgrd_t> holder(new (std::nothrow) afid_mgrd_t());  // freed on every early exit
  afid_mgrd_t *m = holder.get();
  if (!m) return AFID_E_ALLOC;
  const double pi = coarse->pi;
  // CreateMgrdGrid.F90:37-90: uniform y/z, wall-normal grid of type ISTR3R with STR3
  std::vector<double> zcr, zmr, ycr, ymr, xcr;
  afid_hostd::uniform_grid(zcr, zmr, nzmr, in.zlen);
  afid_hostd::uniform_grid(ycr, ymr, nymr, in.ylen);
  if (afid_hostd::x_grid(in.istr3r, nxmr, in.alx3, in.str3, pi, in.pras, xcr) != AFID_OK || in.istr3r == 2) {
    return AFID_E_INVALID;
  }
  const int nxr = nxmr + 1;
  const double dxr = (double)nxmr / in.alx3;
  // CreateMgrdGrid.F90:111-133 (xmr with its two mirror points, g3rmr, udx3mr)
  std::vector<double> xmr_f(nxr + 1, 0.0);  // Fortran xmr(0 .. nxr)
  for (int kc = 1; kc <= nxmr; ++kc) xmr_f[kc] = (xcr[kc - 1] + xcr[kc]) * 0.5;
  xmr_f[0] = 2.0 * xcr[0] - xmr_f[1];
  xmr_f[nxr] = 2.0 * xcr[nxr - 1] - xmr_f[nxmr];
  std::vector<double> g3rmr(nxmr), udx3mr(nxmr), xmr(xmr_f.begin() + 1, xmr_f.begin() + 1 + nxmr);
  for (int kc = 2; kc <= nxmr; ++kc) g3rmr[kc - 1] = (xmr_f[kc + 1] - xmr_f[kc - 1]) * dxr * 0.5;
  g3rmr[0] = (xmr_f[2] - (2 * xcr[0] - xmr_f[1])) * dxr * 0.5;
  for (int kc = 1; kc <= nxmr; ++kc) udx3mr[kc - 1] = dxr / ((xcr[kc] - xcr[kc - 1]) * dxr);
  std::vector<double> ap, ac, am;
  afid_hostd::second_derivative_coeff(ap, ac, am, xmr.data(), nxmr, in.alx3, in.sfixn, in.sfixs);
  // ReadInputFile.F90:109-122
  const double rrho = std::fabs(in.rayt) * in.pras / (std::fabs(in.rays) * in.prat);
  const double bycs = (in.flagsal && in.ffscales == 1) ? 1.0 : 1.0 / rrho;
  const double pecs = coarse->ren * in.pras;
  // SetSalBCs (salinity.F90:105-121)
  if (in.rays >= 0) {
    m->salbp0 = -0.5;
    m->saltp0 = 0.5;
  } else {
    m->salbp0 = 0.5;
    m->saltp0 = -0.5;
  }
  m->salbp.assign((size_t)nymr * nzmr, m->salbp0);
  m->saltp.assign((size_t)nymr * nzmr, m->saltp0);

  // CreateMgrdStencil.F90:1-80
  const std::vector<double> &xc_all = coarse->arr.at("xc"), &xm_all = coarse->arr.at("xm");
  const std::vector<double> xc(xc_all.begin(), xc_all.begin() + nxm + 1), xm(xm_all.begin(), xm_all.begin() + nxm);
  std::vector<double> zc, zm, yc, ym;
  afid_hostd::uniform_grid(zc, zm, nzm, in.zlen);
  afid_hostd::uniform_grid(yc, ym, nym, in.ylen);
  yc.resize(nym);
  zc.resize(nzm);
  const std::vector<int> irangs = interpolation_indices(xm, xmr, in.alx3);
  const std::vector<int> jrangs = interpolation_indices(ym, ymr, in.ylen);
  const std::vector<int> krangs = interpolation_indices(zm, zmr, in.zlen);
  m->w[0] = construct_stencil(xm, xmr, in.alx3, irangs, 'x');
  m->w[1] = construct_stencil(ym, ymr, in.ylen, jrangs, 'y');
  m->w[2] = construct_stencil(zm, zmr, in.zlen, krangs, 'z');
  bool ok = starts_from_intervals(irangs, nxmr, 0, nxm, m->start[0]) &&
            starts_from_intervals(jrangs, nymr, 0, nym, m->start[1]) &&
            starts_from_intervals(krangs, nzmr, 0, nzm, m->start[2]);
  m->fast = (xmr[0] < xm[0] && xmr[nxmr - 1] > xm[nxm - 1]) ? 1 : 0;  // salinity.F90:485
  if (m->fast) {
    // interpolate_xyz_to_coarse_fast: target kc reads refined rows rang(kc)-2 .. rang(kc)+1
    const std::vector<double> *grids_new[3] = {&xc, &yc, &zc};
    const std::vector<double> *grids_ref[3] = {&xmr, &ymr, &zmr};
    const std::vector<double> *grids_c[3] = {&xm, &ym, &zm};
    const std::vector<int> *rangs[3] = {&irangs, &jrangs, &krangs};
    const double lens[3] = {in.alx3, in.ylen, in.zlen};
    const char axes[3] = {'x', 'y', 'z'};
    const int nc[3] = {nxm, nym, nzm};
    for (int d = 0; d < 3; ++d) {
      std::vector<int> rangb;
      std::vector<double> wsal;
      if (in.gaxis == d + 1) {  // to the faces along gravity
        const std::vector<int> range = interpolation_indices(*grids_ref[d], *grids_new[d], lens[d]);
        wsal = construct_stencil(*grids_ref[d], *grids_new[d], lens[d], range, axes[d]);
        rangb = interpolation_indices(*grids_new[d], *grids_ref[d], lens[d]);
      } else {                  // to the cell centres (the cxphic stencils)
        const std::vector<int> ranger = interpolation_indices(*grids_ref[d], *grids_c[d], lens[d]);
        wsal = construct_stencil(*grids_ref[d], *grids_c[d], lens[d], ranger, axes[d]);
        rangb = *rangs[d];
      }
      wsal.resize((size_t)4 * nc[d]);
      m->w[3 + d] = wsal;
      m->start[3 + d].assign(nc[d], 0);
      for (int k = 1; k <= nc[d]; ++k) m->start[3 + d][k - 1] = rangb[k] - 3;
    }
  } else {
    // interpolate_xyz_to_coarse: intervals kcr = 0..nxmr cover the coarse cell centres
    const std::vector<int> irangr = interpolation_indices(xmr, xm, in.alx3);
    const std::vector<int> jrangr = interpolation_indices(ymr, ym, in.ylen);
    const std::vector<int> krangr = interpolation_indices(zmr, zm, in.zlen);
    m->w[3] = construct_stencil(xmr, xm, in.alx3, irangr, 'x');
    m->w[4] = construct_stencil(ymr, ym, in.ylen, jrangr, 'y');
    m->w[5] = construct_stencil(zmr, zm, in.zlen, krangr, 'z');
    ok = ok && starts_from_intervals(irangr, nxm, 0, nxmr, m->start[3]) &&
         starts_from_intervals(jrangr, nym, 0, nymr, m->start[4]) &&
         starts_from_intervals(krangr, nzm, 0, nzmr, m->start[5]);
  }
  if (!ok) {
    return AFID_E_INVALID;
  }
  m->arr["xcr"] = xcr;
  m->arr["xmr"] = xmr;
  m->arr["ymr"] = ymr;
  m->arr["zmr"] = zmr;
  m->arr["g3rmr"] = g3rmr;
  m->arr["udx3mr"] = udx3mr;
  m->arr["ap3sskr"] = ap;
  m->arr["ac3sskr"] = ac;
  m->arr["am3sskr"] = am;
  const char *wn[6] = {"w_to_ref_x", "w_to_ref_y", "w_to_ref_z", "w_to_coarse_x", "w_to_coarse_y", "w_to_coarse_z"};
  const char *sn[6] = {"start_to_ref_x", "start_to_ref_y", "start_to_ref_z", "start_to_coarse_x",
                       "start_to_coarse_y", "start_to_coarse_z"};
  for (int d = 0; d < 6; ++d) {
    m->arr[wn[d]] = m->w[d];
    m->arr[sn[d]] = std::vector<double>(m->start[d].begin(), m->start[d].end());
  }
  m->active_t = in.active_t;
  m->gaxis = in.gaxis;
  afid_sal_grid_t &v = m->view;
  v.nxmr = nxmr;
  v.nymr = nymr;
  v.nzmr = nzmr;
  v.dxr = dxr;
  v.dyr = (double)nymr / in.ylen;
  v.dzr = (double)nzmr / in.zlen;
  v.pecs = pecs;
  v.bycs = bycs;
  v.active_s = in.active_s;
  v.sfixs = in.sfixs;
  v.sfixn = in.sfixn;
  v.xcr = m->arr["xcr"].data();
  v.udx3mr = m->arr["udx3mr"].data();
  v.g3rmr = m->arr["g3rmr"].data();
  v.ap3sskr = m->arr["ap3sskr"].data();
  v.ac3sskr = m->arr["ac3sskr"].data();
  v.am3sskr = m->arr["am3sskr"].data();
  v.salbp = m->salbp.data();
  v.saltp = m->saltp.data();
  for (int d = 0; d < 3; ++d) {
    v.to_ref[d] = afid_stencil_t{(int)m->start[d].size(), m->start[d].data(), m->w[d].data()};
    v.to_coarse[d] = afid_stencil_t{(int)m->start[3 + d].size(), m->start[3 + d].data(), m->w[3 + d].data()};
  }
  *out = holder.release();
  return AFID_OK;
}

void afid_mgrd_destroy(afid_mgrd_t *m) { delete m; }

const afid_sal_grid_t *afid_mgrd_view(const afid_mgrd_t *m) { return m ? &m->view : nullptr; }

int afid_mgrd_fast(const afid_mgrd_t *m) { return m ? m->fast : 0; }

const double *afid_mgrd_array(const afid_mgrd_t *m, const char *name, int *len) {
  if (!m || !name) return nullptr;
  auto it = m->arr.find(name);
  if (it == m->arr.end()) return nullptr;
  if (len) *len = (int)it->second.size();
  return it->second.data();
}

int afid_initial_salinity(const afid_mgrd_t *m, uint64_t seed, double amp, double *sal, int ld_x, int ld_y) {
  return afid_guard([&]() -> int {
    if (!m || !sal) return AFID_E_INVALID;
    const afid_sal_grid_t &v = m->view;
    if (ld_x < v.nxmr || ld_y < v.nymr) return AFID_E_INVALID;
    const std::vector<double> &xmr = m->arr.at("xmr"), &xcr = m->arr.at("xcr");
    const bool ddc = v.active_s == 1 && m->active_t == 1 && m->gaxis == 1;  // salinity.F90:148-157
    const uint64_t nxr = (uint64_t)v.nxmr + 1;
    for (int i = 0; i < v.nzmr; ++i)
      for (int j = 0; j < v.nymr; ++j) {
        double *col = sal + ((size_t)i * ld_y + j) * ld_x;
        for (int k = 0; k < v.nxmr; ++k) {
          if (ddc) {
            col[k] = 0.5 * std::pow(2 * (xmr[k] - 0.5), 7);
            continue;
          }
          // SetLinearSalinity + AddSalinityNoise(amp, localised = .false.) (salinity.F90:176-266)
          const double s0 = m->salbp0 - (m->salbp0 - m->saltp0) * xmr[k] / xcr[v.nxmr];
          const double u = philox_u(seed, (uint64_t)k + nxr * ((uint64_t)j + (uint64_t)v.nymr * i));
          if (std::fabs(s0) + amp > 0.5)
            col[k] = s0 + (0.5 - std::fabs(s0)) * (2.0 * u - 1.0);
          else
            col[k] = s0 + amp * (2.0 * u - 1.0);
        }
      }
    return AFID_OK;
  });
}

}  // extern "C"
