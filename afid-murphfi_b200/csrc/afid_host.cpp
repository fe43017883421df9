// afid_host.cpp — host-side set-up and step control around the GPU substep (include/afid_host.h).
#include "afid_host.h"

#include "afid_continua.h"
#include "afid_host_internal.h"
#include "afid_salinity.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <vector>

namespace {

// ------------------------------------------------------------------------------------------
// bou.in: a title line, a header line, then value lines each preceded by three lines (blank,
// title, header) — the read sequence of ReadInputFile.F90:21-75.
// ------------------------------------------------------------------------------------------
struct LineReader {
  std::vector<std::string> lines;
  size_t pos = 0;
  bool ok = true;
  explicit LineReader(const char *text) {
    std::stringstream ss(text);
    std::string l;
    while (std::getline(ss, l)) lines.push_back(l);
  }
  void skip(int n) { pos += n; }
  std::vector<double> vals(size_t need) {
    std::vector<double> v;
    if (pos >= lines.size()) { ok = false; return std::vector<double>(need, 0.0); }
    std::stringstream ss(lines[pos++]);
    std::string tok;
    while (ss >> tok) {
      for (auto &c : tok)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran double exponent
      char *end = nullptr;
      double x = std::strtod(tok.c_str(), &end);
      if (end == tok.c_str()) break;
      v.push_back(x);
    }
    if (v.size() < need) { ok = false; v.resize(need, 0.0); }
    return v;
  }
};

}  // namespace


namespace afid_hostd {

double philox_u(uint64_t seed, uint64_t n) {
  // Philox4x32-10 (Salmon et al., SC'11): counter (n lo, n hi, 0, 0), key (seed lo, seed hi)
  uint32_t c0 = (uint32_t)n, c1 = (uint32_t)(n >> 32), c2 = 0, c3 = 0;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  const uint64_t bits = ((uint64_t)c0 << 21) | ((uint64_t)c1 >> 11);
  return (double)bits * (1.0 / 9007199254740992.0);
}

void uniform_grid(std::vector<double> &c, std::vector<double> &m, int nm, double len) {
  c.assign(nm + 1, 0.0);
  m.assign(nm, 0.0);
  for (int i = 1; i <= nm + 1; ++i) c[i - 1] = len * (double)(i - 1) / (double)nm;  // grid.F90:19-21
  for (int i = 1; i <= nm; ++i) m[i - 1] = 0.5 * (c[i - 1] + c[i]);
}

void second_derivative_coeff(std::vector<double> &ap3, std::vector<double> &ac3,
                                    std::vector<double> &am3, const double *x, int n, double xlen,
                                    int fix_up, int fix_low) {
  // grid.F90:264-307
  ap3.assign(n, 0.0);
  ac3.assign(n, 0.0);
  am3.assign(n, 0.0);
  int k = 0;
  double a33 = 2.0 / (x[k] + x[k + 1]);
  ap3[k] = a33 / (x[k + 1] - x[k]);
  am3[k] = 0.0;
  if (x[k] == 0.0) {
    ap3[k] = 0.0;
    ac3[k] = 1.0;
  } else {
    ac3[k] = -ap3[k] - fix_low * a33 / x[k];
  }
  for (k = 1; k < n - 1; ++k) {
    a33 = 2.0 / (x[k + 1] - x[k - 1]);
    ap3[k] = a33 / (x[k + 1] - x[k]);
    am3[k] = a33 / (x[k] - x[k - 1]);
    ac3[k] = -ap3[k] - am3[k];
  }
  k = n - 1;
  a33 = 2.0 / (2.0 * xlen - x[k] - x[k - 1]);
  ap3[k] = 0.0;
  am3[k] = a33 / (x[k] - x[k - 1]);
  if (x[k] == xlen) {
    am3[k] = 0.0;
    ac3[k] = 1.0;
  } else {
    ac3[k] = -am3[k] - fix_up * a33 / (xlen - x[k]);
  }
}

// Wall-normal faces xc[0..nxm] of grid type istr3 (grid.F90); schmidt enters ISTR3 = 3 only
// (1 on the coarse grid, CreateGrid.F90:70; PraS on the refined grid, CreateMgrdGrid.F90:64).
int x_grid(int istr3, int nxm, double L, double s, double pi, double schmidt, std::vector<double> &xc) {
  const int nx = nxm + 1;
  switch (istr3) {
    case 0: {
      std::vector<double> xmv;
      uniform_grid(xc, xmv, nxm, L);
      break;
    }
    case 1: {  // grid.F90:133-151
      xc.assign(nx, 0.0);
      for (int i = 2; i <= nxm; ++i) {
        const double q = 2.0 * (i - 1) / nxm - 1;
        xc[i - 1] = L / 2.0 * (s * std::pow(q, 7) + 2.0 * (i - 1) / nxm - 1) / (s + 1) + L / 2.0;
      }
      xc[nxm] = L;
      break;
    }
    case 2:
    case 3: {  // grid.F90:153-213 (natural boundary-layer stretching)
      const double jb = 16.0, c_eta = 0.8, alpha = 1.5, dyw = 0.1;
      xc.assign(nx, 0.0);
      if (istr3 == 2) {
        for (int j = 1; j <= nxm + 1; ++j) {
          const double jm = j - 1;
          xc[j - 1] = 1 / (1.0 + (jm / jb) * (jm / jb)) *
                      (dyw * jm + std::pow(0.75 * alpha * c_eta * jm, 4.0 / 3.0) * (jm / jb) * (jm / jb));
        }
      } else {
        const int nh = nxm / 2;
        for (int j = 1; j <= nh + 1; ++j) {
          const double jm = j - 1;
          xc[j - 1] = 1 / (1.0 + (jm / jb) * (jm / jb)) *
                      (dyw * jm + std::pow(0.75 * alpha * c_eta * jm / std::pow(schmidt, 0.5), 4.0 / 3.0) *
                                      (jm / jb) * (jm / jb));
        }
        const double lh = 2.0 * xc[nh];
        for (int j = 1; j <= nh; ++j) xc[nxm + 1 - j] = lh - xc[j - 1];
      }
      const double top = xc[nxm];
      for (auto &v : xc) v = v / top * L;
      break;
    }
    case 4: {  // grid.F90:29-53
      const double tstr = std::tanh(s);
      xc.assign(nx, 0.0);
      for (int i = 2; i <= nxm + 1; ++i) {
        const double z2 = (double)(2 * (i - 1) - nxm) / (double)nxm;
        xc[i - 1] = 0.5 * (1 + std::tanh(s * z2) / tstr) * L;
        if (xc[i - 1] < 0.0 || xc[i - 1] > L) return AFID_E_INVALID;
      }
      break;
    }
    case 6:
    case 7: {  // grid.F90:55-131 (clipped Chebyshev)
      const int nclip = (int)s;
      const int n_ext = (istr3 == 6) ? nxm + 1 + 2 * nclip : nxm + 1 + nclip;
      std::vector<double> etazm(n_ext), etaz(nx);
      for (int i = 1; i <= n_ext; ++i)
        etazm[i - 1] = (istr3 == 6) ? std::cos(pi * ((double)i - 0.5) / (double)n_ext)
                                        : std::cos(pi * (double)i / (double)n_ext / 2.0);
      for (int i = 1; i <= nx; ++i) etaz[i - 1] = etazm[i + nclip - 1];
      xc.assign(nx, 0.0);
      if (istr3 == 6) {
        const double delet = etaz[0] - etaz[nxm];
        for (auto &v : etaz) v = 2.0 * v / delet;
        for (int i = 2; i <= nxm; ++i) xc[i - 1] = 0.5 * L * (1.0 - etaz[i - 1]);
      } else {
        const double delet = etaz[0];
        for (auto &v : etaz) v = v / delet;
        for (int i = 2; i <= nxm; ++i) xc[i - 1] = L * (1.0 - etaz[i - 1]);
      }
      xc[nxm] = L;
      break;
    }
    default:
      return AFID_E_INVALID;
  }
  return AFID_OK;
}

}  // namespace afid_hostd

using afid_hostd::philox_u;
using afid_hostd::second_derivative_coeff;
using afid_hostd::uniform_grid;

namespace {

// The mean-profile samples and movie cuts afid_run_io collects for means.h5 and flowmov/.
struct Samples {
  std::vector<double> ptimes, prof, salprof, ftimes;
  size_t dropped = 0;  // movie frames left out once the plane buffer is full
  std::vector<double> planes[3], salplanes[3];
  std::vector<double> mplanes[3], salmplanes[3];  // mean_yplane / mean_zplane (axis 1, 2)

  int profiles(afid_ctx_t *ctx, const afid_input_t *in, const afid_mgrd_t *mg, double time) {
    const size_t off = prof.size();
    prof.resize(off + (size_t)AFID_NUM_PROFILES * in->nxm);
    int r = afid_gpu_mean_profiles(ctx, prof.data() + off);
    if (r == AFID_OK && mg) {
      const size_t o2 = salprof.size();
      salprof.resize(o2 + (size_t)AFID_NUM_SAL_PROFILES * afid_mgrd_view(mg)->nxmr);
      r = afid_gpu_sal_profiles(ctx, salprof.data() + o2);
    }
    ptimes.push_back(time);
    return r;
  }

  // The cut positions of MakeMovie{X,Y,Z}Cut.F90 (0-based): x at 0 (vx at 1; nxm/2 - 1 and
  // max(nxm/2, 2) - 1 when RAYS and RAYT are both negative), y at nym/2, z at nzm/2; the refined
  // salinity likewise, cut on the host from a download of the field.
  // The planes are kept in host memory until the run ends; past kMovieBytes further frames are
  // not collected (the reference appends each frame to its files instead).
  static constexpr size_t kMovieBytes = size_t(2) << 30;

  int movie(afid_ctx_t *ctx, const afid_input_t *in, const afid_mgrd_t *mg, double time) {
    const bool both_neg = in->rays < 0 && in->rayt < 0;
    const int icx = both_neg ? in->nxm / 2 : 1, nx = in->nxm + 1;
    const size_t psz[3] = {(size_t)in->nzm * in->nym, (size_t)in->nzm * nx, (size_t)in->nym * nx};
    const bool means = in->nym > 1 && in->nzm > 1;  // write_mean_planes (main.F90:42)
    size_t frame_bytes = 4 * (psz[0] + psz[1] + psz[2] + (means ? psz[1] + psz[2] : 0)) * sizeof(double);
    if (mg) {
      const afid_sal_grid_t *v = afid_mgrd_view(mg);
      frame_bytes += ((size_t)v->nzmr * v->nymr + (size_t)v->nzmr * v->nxmr + (size_t)v->nymr * v->nxmr) * sizeof(double);
      if (means) frame_bytes += ((size_t)v->nzmr * v->nxmr + (size_t)v->nymr * v->nxmr) * sizeof(double);
    }
    if ((ftimes.size() + 1) * frame_bytes > kMovieBytes) {
      // the frame is not kept: say so once, and count the frames left out
      if (dropped++ == 0)
        std::fprintf(stderr,
                     "afid_run_io: movie planes exceed %zu bytes at time %.6g; this and later frames "
                     "are not written to flowmov/\n",
                     kMovieBytes, time);
      return AFID_OK;
    }
    for (int axis = 0; axis < 3; ++axis)
      for (int which = 0; which < 4; ++which) {
        const int idx = axis == 0 ? (which == 0 ? std::max(icx, 2) - 1 : icx - 1) : axis == 1 ? in->nym / 2 : in->nzm / 2;
        const size_t off = planes[axis].size();
        planes[axis].resize(off + psz[axis]);
        const int r = afid_gpu_slice(ctx, which, axis, idx, planes[axis].data() + off);
        if (r != AFID_OK) return r;
      }
    // mean_yplane / mean_zplane beside the cuts (main.F90:340-343)
    for (int axis = 1; means && axis <= 2; ++axis) {
      for (int which = 0; which < 4; ++which) {
        const size_t off = mplanes[axis].size();
        mplanes[axis].resize(off + psz[axis]);
        const int r = afid_gpu_mean_plane(ctx, which, axis, mplanes[axis].data() + off);
        if (r != AFID_OK) return r;
      }
      if (mg) {
        const afid_sal_grid_t *v = afid_mgrd_view(mg);
        const size_t off = salmplanes[axis].size();
        salmplanes[axis].resize(off + (size_t)(axis == 1 ? v->nzmr : v->nymr) * v->nxmr);
        const int r = afid_gpu_sal_mean_plane(ctx, axis, salmplanes[axis].data() + off);
        if (r != AFID_OK) return r;
      }
    }
    if (mg) {
      const afid_sal_grid_t *v = afid_mgrd_view(mg);
      const int nxmr = v->nxmr, nymr = v->nymr, nzmr = v->nzmr;
      std::vector<double> sal((size_t)nxmr * nymr * nzmr);
      const int r = afid_gpu_sal_download(ctx, sal.data(), nxmr, nymr);
      if (r != AFID_OK) return r;
      const int ix = (both_neg ? nxmr / 2 : 1) - 1, iy = nymr / 2, iz = nzmr / 2;
      for (int i = 0; i < nzmr; ++i)
        for (int j = 0; j < nymr; ++j) salplanes[0].push_back(sal[((size_t)i * nymr + j) * nxmr + ix]);
      for (int i = 0; i < nzmr; ++i)
        for (int k = 0; k < nxmr; ++k) salplanes[1].push_back(sal[((size_t)i * nymr + iy) * nxmr + k]);
      for (int j = 0; j < nymr; ++j)
        for (int k = 0; k < nxmr; ++k) salplanes[2].push_back(sal[((size_t)iz * nymr + j) * nxmr + k]);
    }
    ftimes.push_back(time);
    return AFID_OK;
  }

  int write(const char *dir, const afid_input_t *in, const afid_mgrd_t *mg) const {
    const afid_sal_grid_t *v = mg ? afid_mgrd_view(mg) : nullptr;
    int r = AFID_OK;
    if (in->tout > 0.0 && !ptimes.empty()) {
      // samples whose number nint(time / TOUT) is out of the five-digit range are dropped; of
      // two samples with the same number afid_write_means keeps the later one, as the
      // reference's writer deletes and rewrites the dataset
      std::vector<double> t, p, q;
      const size_t np = (size_t)AFID_NUM_PROFILES * in->nxm, nq = v ? (size_t)AFID_NUM_SAL_PROFILES * v->nxmr : 0;
      for (size_t k = 0; k < ptimes.size(); ++k) {
        const double fr = std::round(ptimes[k] / in->tout);
        if (!(fr >= 0.0 && fr <= 99999.0)) continue;
        t.push_back(ptimes[k]);
        p.insert(p.end(), prof.begin() + k * np, prof.begin() + (k + 1) * np);
        if (v) q.insert(q.end(), salprof.begin() + k * nq, salprof.begin() + (k + 1) * nq);
      }
      r = afid_write_means(dir, in->tout, (int)t.size(), t.data(), in->nxm, p.data(), v ? v->nxmr : 0,
                           v ? q.data() : nullptr);
    }
    if (dropped)
      std::fprintf(stderr, "afid_run_io: %zu movie frames were left out of flowmov/ (plane buffer full)\n", dropped);
    if (r != AFID_OK || !(in->tframe > 0.0) || ftimes.empty()) return r;
    for (size_t f = 0; f < ftimes.size(); ++f)
      if (!(std::round(ftimes[f] / in->tframe) >= 0.0 && std::round(ftimes[f] / in->tframe) <= 99999.0)) return r;
    for (int axis = 0; axis < 3 && r == AFID_OK; ++axis)
      r = afid_write_movie(dir, axis, in->tframe, (int)ftimes.size(), ftimes.data(), in->nxm, in->nym, in->nzm,
                           planes[axis].data(), v ? v->nxmr : 0, v ? v->nymr : 0, v ? v->nzmr : 0,
                           v ? salplanes[axis].data() : nullptr);
    for (int axis = 1; axis <= 2 && r == AFID_OK && in->nym > 1 && in->nzm > 1; ++axis)
      r = afid_write_movie_mean(dir, axis, in->tframe, (int)ftimes.size(), ftimes.data(), in->nxm, in->nym,
                                in->nzm, mplanes[axis].data(), v ? v->nxmr : 0, v ? v->nymr : 0, v ? v->nzmr : 0,
                                v ? salmplanes[axis].data() : nullptr);
    return r;
  }
};

}  // namespace

extern "C" {

int afid_parse_bou_in(const char *text, afid_input_t *o) {
  return afid_guard([&]() -> int {
    if (!text || !o) return AFID_E_INVALID;
    std::memset(o, 0, sizeof(*o));
    LineReader r(text);
    r.skip(2);
    auto v = r.vals(4);
    o->nxm = (int)v[0]; o->nym = (int)v[1]; o->nzm = (int)v[2]; o->nsst = (int)v[3];
    r.skip(3);
    v = r.vals(4);
    o->multires = (int)v[0]; o->nxmr = (int)v[1]; o->nymr = (int)v[2]; o->nzmr = (int)v[3];
    r.skip(3);
    v = r.vals(2);
    o->flagsal = (int)v[0]; o->flagpf = (int)v[1];
    r.skip(3);
    v = r.vals(2);
    o->nread = (int)v[0]; o->ireset = (int)v[1];
    r.skip(3);
    v = r.vals(3);
    o->ntst = (int)v[0]; o->walltimemax = v[1]; o->tmax = v[2];
    r.skip(3);
    v = r.vals(3);
    o->tout = v[0]; o->tframe = v[1]; o->save_3d = v[2];
    r.skip(3);
    v = r.vals(3);
    o->alx3 = v[0]; o->ylen = v[1]; o->zlen = v[2];
    r.skip(3);
    v = r.vals(3);
    o->istr3 = (int)v[0]; o->str3 = v[1]; o->istr3r = (int)v[2];
    r.skip(3);
    v = r.vals(5);
    o->rayt = v[0]; o->prat = v[1]; o->rays = v[2]; o->pras = v[3]; o->ffscales = (int)v[4];
    r.skip(3);
    v = r.vals(6);
    o->idtv = (int)v[0]; o->dt = v[1]; o->resid = v[2]; o->limit_cfl = v[3]; o->dtmin = v[4]; o->dtmax = v[5];
    r.skip(3);
    v = r.vals(6);
    o->inslws = (int)v[0]; o->inslwn = (int)v[1]; o->tfixs = (int)v[2]; o->tfixn = (int)v[3];
    o->sfixs = (int)v[4]; o->sfixn = (int)v[5];
    r.skip(3);
    v = r.vals(3);
    o->active_t = (int)v[0]; o->active_s = (int)v[1]; o->gaxis = (int)v[2];
    r.skip(3);
    v = r.vals(5);
    o->xplusu = v[0]; o->xminusu = v[1]; o->dpdy = v[2]; o->dpdz = v[3]; o->melt = (int)v[4];
    if (!r.ok) return AFID_E_INVALID;
    if (o->nxm < 1 || o->nym < 1 || o->nzm < 1) return AFID_E_INVALID;
    return AFID_OK;
  });
}

int afid_read_bou_in(const char *path, afid_input_t *out) {
  return afid_guard([&]() -> int {
    if (!path) return AFID_E_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return AFID_E_INVALID;
    std::string s;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
    std::fclose(f);
    return afid_parse_bou_in(s.c_str(), out);
  });
}

static int tables_create(const afid_input_t *in, int precision, afid_tables_t **out);

int afid_tables_create(const afid_input_t *in, int precision, afid_tables_t **out) {
  if (!in || !out) return AFID_E_INVALID;
  *out = nullptr;
  // sizes far beyond any grid one GPU can hold are input errors, not allocation requests (the
  // host tables include two y-z planes of plate temperatures)
  if (in->nxm < 2 || in->nym < 1 || in->nzm < 1 || in->nxm > (1 << 20) || in->nym > (1 << 20) ||
      in->nzm > (1 << 20) || (long long)in->nym * in->nzm > (1LL << 28))
    return AFID_E_INVALID;
  try {
    return tables_create(in, precision, out);
  } catch (const std::bad_alloc &) {
    return AFID_E_ALLOC;
  }
}

static int tables_create(const afid_input_t *in, int precision, afid_tables_t **out) {
  std::unique_ptr<afid_tables_t> holder(new (std::nothrow) afid_tables_t());  // freed on every early exit
  afid_tables_t *t = holder.get();
  if (!t) return AFID_E_ALLOC;
  t->in = *in;
  const int nxm = in->nxm, nym = in->nym, nzm = in->nzm, nx = nxm + 1;
  // ReadInputFile.F90:109-123
  const double rrho = std::fabs(in->rayt) * in->pras / (std::fabs(in->rays) * in->prat);
  if (in->flagsal && in->ffscales == 1) {
    t->ren = std::sqrt(std::fabs(in->rays) / in->pras);
    t->byct = rrho;
  } else {
    t->ren = std::sqrt(std::fabs(in->rayt) / in->prat);
    t->byct = 1.0;
  }
  t->pect = t->ren * in->prat;
  t->pi = 2.0 * std::asin(1.0);
  const double pi = t->pi;

  std::vector<double> zc, zm, yc, ym, xc;
  uniform_grid(zc, zm, nzm, in->zlen);
  uniform_grid(yc, ym, nym, in->ylen);
  if (afid_hostd::x_grid(in->istr3, nxm, in->alx3, in->str3, pi, 1.0, xc) != AFID_OK) {
    return AFID_E_INVALID;  // ISTR3=5 (scallop, channel-flow specific) is not on this path
  }
  // CreateGrid.F90:100-138
  const double dx = (double)nxm / in->alx3, dy = (double)nym / in->ylen, dz = (double)nzm / in->zlen;
  t->dx = dx;
  t->dy = dy;
  t->dz = dz;
  std::vector<double> xm(nx, 0.0), g3rc(nx, 0.0), g3rm(nx, 0.0), d3xc(nx, 0.0), d3xm(nx, 0.0),
      udx3m(nx, 0.0), udx3c(nx, 0.0);
  for (int kc = 0; kc < nxm; ++kc) xm[kc] = (xc[kc] + xc[kc + 1]) * 0.5;
  xm[nx - 1] = 2 * xc[nx - 1] - xm[nxm - 1];
  for (int kc = 1; kc < nxm; ++kc) {
    g3rc[kc] = (xc[kc + 1] - xc[kc - 1]) * dx * 0.5;
    g3rm[kc] = (xm[kc + 1] - xm[kc - 1]) * dx * 0.5;
  }
  g3rm[0] = (xm[1] - (2 * xc[0] - xm[0])) * dx * 0.5;
  g3rc[0] = (xc[1] - xc[0]) * dx;
  g3rc[nx - 1] = (xc[nx - 1] - xc[nxm - 1]) * dx;
  for (int kc = 0; kc < nxm; ++kc) {
    d3xc[kc] = (xc[kc + 1] - xc[kc]) * dx;
    d3xm[kc] = (xm[kc + 1] - xm[kc]) * dx;
  }
  for (int kc = 0; kc < nxm; ++kc) {
    udx3m[kc] = dx / d3xc[kc];
    udx3c[kc] = dx / g3rc[kc];
  }
  udx3c[nx - 1] = dx / g3rc[nx - 1];
  std::vector<double> ap3ck, ac3ck, am3ck, ap3sk, ac3sk, am3sk, ap3ssk, ac3ssk, am3ssk;
  second_derivative_coeff(ap3ck, ac3ck, am3ck, xc.data(), nx, in->alx3, 1, 1);
  second_derivative_coeff(ap3sk, ac3sk, am3sk, xm.data(), nxm, in->alx3, in->inslwn, in->inslws);
  second_derivative_coeff(ap3ssk, ac3ssk, am3ssk, xm.data(), nxm, in->alx3, in->tfixn, in->tfixs);
  // pressure.F90:68-114
  std::vector<double> ak1(nzm), ak2(nym);
  const int nzmh = nzm / 2 + 1, nymh = nym / 2 + 1;
  for (int i = 1; i <= nzm; ++i) {
    const double ao = (i <= nzmh) ? (i - 1) * 2.0 * pi : -(nzm - i + 1) * 2.0 * pi;
    ak1[i - 1] = 2.0 * (1.0 - std::cos(ao / nzm)) * std::pow((double)nzm / in->zlen, 2);
  }
  for (int j = 1; j <= nym; ++j) {
    const double ap = (j <= nymh) ? (j - 1) * 2.0 * pi : -(nym - j + 1) * 2.0 * pi;
    ak2[j - 1] = 2.0 * (1.0 - std::cos(ap / nym)) * std::pow((double)nym / in->ylen, 2);
  }
  const double dxq = dx * dx;
  std::vector<double> amphk(nx, 0.0), acphk(nx, 0.0), apphk(nx, 0.0);
  for (int kc = 0; kc < nxm; ++kc) {
    const int km = (kc == 0) ? 0 : kc - 1;
    const int kp = (kc == nxm - 1) ? kc : kc + 1;
    const int kmc = kc - km, kpc = kp - kc;
    const double a33icc = kmc * dxq / d3xm[km];
    const double a33icp = kpc * dxq / d3xm[kc];
    const double ugmmm = 1.0 / d3xc[kc];
    amphk[kc] = a33icc * ugmmm;
    apphk[kc] = a33icp * ugmmm;
    acphk[kc] = -(amphk[kc] + apphk[kc]);
  }
  auto &A = t->arr;
  A["xc"] = xc;
  A["xm"] = xm;
  A["yc"] = yc;
  A["ym"] = ym;
  A["zc"] = zc;
  A["zm"] = zm;
  A["g3rc"] = g3rc;
  A["g3rm"] = g3rm;
  A["d3xc"] = d3xc;
  A["d3xm"] = d3xm;
  A["udx3c"] = udx3c;
  A["udx3m"] = udx3m;
  A["ap3ck"] = ap3ck;
  A["ac3ck"] = ac3ck;
  A["am3ck"] = am3ck;
  A["ap3sk"] = ap3sk;
  A["ac3sk"] = ac3sk;
  A["am3sk"] = am3sk;
  A["ap3ssk"] = ap3ssk;
  A["ac3ssk"] = ac3ssk;
  A["am3ssk"] = am3ssk;
  A["ak1"] = ak1;
  A["ak2"] = ak2;
  A["amphk"] = amphk;
  A["acphk"] = acphk;
  A["apphk"] = apphk;
  // SetTempBCs.F90:18-41
  double top, bot;
  if (in->rayt >= 0) {
    if (in->inslwn == 0) { top = 0.0; bot = 1.0; }
    else { top = -0.5; bot = 0.5; }
  } else {
    top = 0.5;
    bot = -0.5;
  }
  t->tempbp.assign((size_t)nym * nzm, bot);
  t->temptp.assign((size_t)nym * nzm, top);

  afid_grid_t &g = t->grid;
  g.nxm = nxm;
  g.nym = nym;
  g.nzm = nzm;
  g.alx3 = in->alx3;
  g.ylen = in->ylen;
  g.zlen = in->zlen;
  g.xc = A["xc"].data();
  g.xm = A["xm"].data();
  g.g3rc = A["g3rc"].data();
  g.udx3c = A["udx3c"].data();
  g.udx3m = A["udx3m"].data();
  g.ap3ck = A["ap3ck"].data();
  g.ac3ck = A["ac3ck"].data();
  g.am3ck = A["am3ck"].data();
  g.ap3sk = A["ap3sk"].data();
  g.ac3sk = A["ac3sk"].data();
  g.am3sk = A["am3sk"].data();
  g.ap3ssk = A["ap3ssk"].data();
  g.ac3ssk = A["ac3ssk"].data();
  g.am3ssk = A["am3ssk"].data();
  g.amphk = A["amphk"].data();
  g.acphk = A["acphk"].data();
  g.apphk = A["apphk"].data();
  g.ak1 = A["ak1"].data();
  g.ak2 = A["ak2"].data();
  afid_params_t &p = t->params;
  std::memset(&p, 0, sizeof p);
  p.ren = t->ren;
  p.pect = t->pect;
  p.byct = t->byct;
  p.active_t = in->active_t;
  p.gaxis = in->gaxis;
  p.inslws = in->inslws;
  p.inslwn = in->inslwn;
  p.tfixs = in->tfixs;
  p.tfixn = in->tfixn;
  p.xplusu = in->xplusu;
  p.xminusu = in->xminusu;
  p.dpdy = in->dpdy;
  p.dpdz = in->dpdz;
  p.nsst = in->nsst;
  p.precision = precision;
  p.tempbp = t->tempbp.data();
  p.temptp = t->temptp.data();
  *out = holder.release();
  return AFID_OK;
}

void afid_tables_destroy(afid_tables_t *t) { delete t; }
const afid_grid_t *afid_tables_grid(const afid_tables_t *t) { return t ? &t->grid : nullptr; }
const afid_params_t *afid_tables_params(const afid_tables_t *t) { return t ? &t->params : nullptr; }

const double *afid_tables_array(const afid_tables_t *t, const char *name, int *len) {
  if (!t || !name) return nullptr;
  auto it = t->arr.find(name);
  if (it == t->arr.end()) return nullptr;
  if (len) *len = (int)it->second.size();
  return it->second.data();
}

double afid_philox_uniform(uint64_t seed, uint64_t n) { return philox_u(seed, n); }

int afid_initial_temperature(const afid_tables_t *t, uint64_t seed, double eps, double *temp, int ld_x,
                             int ld_y) {
  return afid_guard([&]() -> int {
    if (!t || !temp) return AFID_E_INVALID;
    const int nxm = t->in.nxm, nym = t->in.nym, nzm = t->in.nzm, nx = nxm + 1;
    if (ld_x < nx || ld_y < nym) return AFID_E_INVALID;
    const std::vector<double> &xm = t->arr.at("xm");
    for (int i = 0; i < nzm; ++i)
      for (int j = 0; j < nym; ++j) {
        const double tb = t->tempbp[(size_t)j + (size_t)nym * i], tt = t->temptp[(size_t)j + (size_t)nym * i];
        double *col = temp + ((size_t)i * ld_y + j) * ld_x;
        for (int k = 0; k < nxm; ++k) {
          double v = tb + (tt - tb) * xm[k] / t->in.alx3;  // CreateInitialConditions.F90:178-185
          const double u = philox_u(seed, (uint64_t)k + (uint64_t)nx * ((uint64_t)j + (uint64_t)nym * i));
          const double dist = std::fabs(xm[k] - 0.5);
          const double amp = (dist + eps > 0.5) ? 0.5 - dist : eps;  // :190-196
          col[k] = v + amp * (2.0 * u - 1.0);
        }
      }
    return AFID_OK;
  });
}

int afid_next_dt(const afid_input_t *in, int ntime, double *dt, double cflm, double *cfl_report) {
  return afid_guard([&]() -> int {
    if (!in || !dt) return AFID_E_INVALID;
    int err = 0;
    if (in->idtv == 1) {  // main.F90:287-302
      if (ntime > 1) {
        *dt = (cflm < 1.0e-8) ? in->dtmax : in->limit_cfl / cflm;
        if (*dt > in->dtmax) *dt = in->dtmax;
      }
      if (!(*dt >= in->dtmin)) err = AFID_E_DTMIN;  // also a NaN dt from a NaN CFL
      if (cfl_report) *cfl_report = cflm;
    } else {  // main.F90:297-298
      const double c = cflm * (*dt);
      if (!(c <= in->limit_cfl)) err = AFID_E_CFL;  // also a NaN CFL
      if (cfl_report) *cfl_report = c;
    }
    return err;
  });
}

int afid_run(const afid_input_t *in, int precision, uint64_t seed, int nsteps, int stats_every, afid_step_cb cb,
             void *user, afid_run_stats_t *stats) {
  return afid_guard([&]() -> int {
    return afid_run_io(in, precision, seed, nsteps, stats_every, cb, user, nullptr, stats);
  });
}

int afid_run_io(const afid_input_t *in, int precision, uint64_t seed, int nsteps, int stats_every, afid_step_cb cb,
                void *user, const char *dir, afid_run_stats_t *stats) {
  return afid_guard([&]() -> int {
    if (!in) return AFID_E_INVALID;
    afid_tables_t *t = nullptr;
    int s = afid_tables_create(in, precision, &t);
    if (s != AFID_OK) return s;
    afid_ctx_t *ctx = nullptr;
    s = afid_gpu_create(&t->grid, &t->params, &ctx);
    if (s != AFID_OK) { afid_tables_destroy(t); return s; }
    const int nxm = in->nxm, nym = in->nym, nzm = in->nzm, nx = nxm + 1;
    // multi-resolution salinity (MULTIRES = FLAGSAL = 1): refined grid, CreateInitialSalinity with
    // Philox key seed + 1, and the refined-grid CFL number for the dt rule (main.F90:285-293)
    afid_mgrd_t *mg = nullptr;
    if (in->flagsal) {
      s = afid_mgrd_create(t, &mg);
      if (s == AFID_OK) s = afid_gpu_sal_create(ctx, afid_mgrd_view(mg));
    }
    double time = 0.0;
    afid_continua_master_t master{};
    afid_continua_master_from_input(in, 0.0, &master);
    if (s == AFID_OK && dir && in->nread) {  // ReadFlowInterp (main.F90:157-161)
      s = afid_gpu_read_flow_interp(ctx, dir, in, &time, nullptr);
      if (in->ireset) time = 0.0;           // ReadFlowInterp.F90:173
    } else if (s == AFID_OK) {
      std::vector<double> temp((size_t)nx * nym * nzm, 0.0);
      afid_initial_temperature(t, seed, 1e-3, temp.data(), nx, nym);
      std::vector<double> zero(temp.size(), 0.0);
      s = afid_gpu_upload(ctx, zero.data(), zero.data(), zero.data(), temp.data(), zero.data(), nx, nym);
      if (s == AFID_OK && mg) {
        const afid_sal_grid_t *v = afid_mgrd_view(mg);
        std::vector<double> sal((size_t)v->nxmr * v->nymr * v->nzmr);
        afid_initial_salinity(mg, seed + 1, 5e-3, sal.data(), v->nxmr, v->nymr);
        s = afid_gpu_sal_upload(ctx, sal.data(), v->nxmr, v->nymr);
      }
    }
    // Outputs besides the restart files (dir only): cordin_info.h5 (WriteGridInfo), a mean-profile
    // sample at start-up and at TOUT (CalcMeanProfiles, main.F90:227, 315-320) and the three movie
    // cuts at start-up and at TFRAME (Mkmov_*, main.F90:230-232, 333-341), collected here and
    // written when the run ends
    Samples out;
    const bool outputs = dir != nullptr;
    if (s == AFID_OK && outputs) {
      s = afid_write_grid_info(dir, t, mg);
      if (s == AFID_OK) s = out.profiles(ctx, in, mg, time);
      if (s == AFID_OK) s = out.movie(ctx, in, mg, time);
    }
    // 3-D frames: at start-up (main.F90:241) and when mod(time, SAVE_3D) < dt past the first
    // TFRAME (main.F90:376-381); skipped when SAVE_3D or TFRAME is not positive
    const bool frames = dir && in->save_3d > 0.0 && in->tframe > 0.0;
    if (s == AFID_OK && frames) {
      master.time = time;
      s = afid_gpu_write_flow_field(ctx, dir, 0, in->save_3d, &master);
    }
    afid_run_stats_t st{};
    const int total = (nsteps < 0) ? in->ntst + 1 : nsteps;
    double dt = in->dt;
    const double ra_pr = std::fabs(in->rayt) * in->prat;
    auto t0 = std::chrono::steady_clock::now();
    int errorcode = 0;
    for (int ntime = 0; ntime < total && s == AFID_OK; ++ntime) {
      double cflm = 0.0;
      if ((s = mg ? afid_gpu_sal_cfl(ctx, &cflm) : afid_gpu_cfl(ctx, &cflm)) != AFID_OK) break;
      double cflr = 0.0;
      errorcode = afid_next_dt(in, ntime, &dt, cflm, &cflr);
      if ((s = afid_gpu_timemarcher(ctx, dt, ntime)) != AFID_OK) break;
      time += dt;
      st.steps_done = ntime + 1;
      st.cfl = cflr;
      // main.F90:346-358: divergence check on step 1 and every tout
      if (ntime == 1 || std::fmod(time, in->tout) < dt) {
        double dmax = 0.0;
        if ((s = afid_gpu_divmax(ctx, &dmax)) != AFID_OK) break;
        st.divmax = dmax;
        if (!(std::fabs(dmax) <= in->resid)) errorcode = AFID_E_DIVERGENCE;  // NaN included
      }
      if (stats_every > 0 && cb && ((ntime + 1) % stats_every == 0)) {
        double nu = 0, ke = 0;
        afid_gpu_globals(ctx, ra_pr, &nu, &ke, nullptr);
        cb(ntime, time, dt, nu, ke, user);
      }
      if (outputs && in->tout > 0.0 && std::fmod(time, in->tout) < dt &&
          (s = out.profiles(ctx, in, mg, time)) != AFID_OK)
        break;
      if (outputs && in->tframe > 0.0 && std::fmod(time, in->tframe) < dt && std::floor(time / in->tframe) != 0.0 &&
          (s = out.movie(ctx, in, mg, time)) != AFID_OK)
        break;
      if (frames && std::fmod(time, in->save_3d) < dt && std::floor(time / in->tframe) != 0.0) {
        master.time = time;
        if ((s = afid_gpu_write_flow_field(ctx, dir, 0, in->save_3d, &master)) != AFID_OK) break;
      }
      if (time > in->tmax) errorcode = 333;
      if (errorcode == 0 && nsteps < 0 && ntime == in->ntst) errorcode = 555;
      if (errorcode != 0) break;
    }
    if (s == AFID_OK) s = afid_gpu_synchronize(ctx);
    auto t1 = std::chrono::steady_clock::now();
    st.seconds = std::chrono::duration<double>(t1 - t0).count();
    st.time = time;
    st.dt = dt;
    st.errorcode = errorcode;
    if (s == AFID_OK) afid_gpu_globals(ctx, ra_pr, &st.nu_vol, &st.ke, nullptr);
    // QuitRoutine.F90:37: the continua files on a normal exit
    if (s == AFID_OK && dir && (errorcode == 0 || errorcode == 333 || errorcode == 334 || errorcode == 555)) {
      master.time = time;
      s = afid_gpu_write_flow_field(ctx, dir, 1, in->save_3d, &master);
    }
    // means.h5 and the movie files hold every sample taken, as the reference's files would
    if (s == AFID_OK && outputs) s = out.write(dir, in, mg);
    if (stats) *stats = st;
    afid_gpu_destroy(ctx);
    afid_mgrd_destroy(mg);
    afid_tables_destroy(t);
    return s;
  });
}

}  // extern "C"
