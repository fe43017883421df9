// afid_stats.cu — on-device statistics and outputs: the wall-normal profiles of
// CalcMeanProfiles.F90, the spectra of spectra.F90 and the movie planes of MakeMovie*Cut.F90.
//
// The fifteen y-z averages written to means.h5 (Tbar, vybar, vzbar, vxT, vyT, vzT, Trms, vxrms,
// vyrms, vzrms, vxvy, vxvz, vyvz, chiT, epsilon) are reduced in two passes: every block walks a
// strided set of x-columns with one thread per wall-normal row k and keeps the fifteen running
// sums in registers, writes them as one partial row per block, and a second kernel adds the
// partials in block order (deterministic, no atomics).  The host applies the reference's
// normalisation (CalcMeanProfiles.F90:88-102, 203-207).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "afid_internal.h"

namespace afid {

constexpr int kNumProfiles = 15;

// Sums over the columns [col0, col0 + ncols) of the fifteen integrands of
// CalcMeanProfiles.F90:48-72 (means and second moments), :104-128 (chiT) and :164-199
// (epsilon).  Block = one thread per row k (blockDim.x >= nxm); partial[(b*15 + q)*nxm + k].
__global__ void __launch_bounds__(1024)
    k_mean_partial(Geom g0, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                   const double *__restrict__ vz, const double *__restrict__ temp, int col0, int ncols,
                   double *__restrict__ partial) {
  const int k = threadIdx.x;
  const int nxm = g0.nxm;
  double acc[kNumProfiles];
#pragma unroll
  for (int q = 0; q < kNumProfiles; ++q) acc[q] = 0.0;
  if (k < nxm) {
    const int kp = k + 1, km = k - 1;
    const bool lo = (k == 0), hi = (k == nxm - 1);
    const double udx3m = __ldg(t.udx3m + k);
    const double tdx = 0.5 * g0.dx / __ldg(t.g3rm + k);                       // :113-126
    const double tdx2 = 0.125 * (g0.dx / __ldg(t.g3rm + k)) * (g0.dx / __ldg(t.g3rm + k));  // :182-197
    for (int cc = blockIdx.x; cc < ncols; cc += gridDim.x) {
      const int col = col0 + cc;
      const int j = col % g0.nym, i = col / g0.nym;
      Geom g = g0;
      bind_instance(g, i);
      const int jp = wrap_inc(j, g.nym), jm = wrap_dec(j, g.nym);
      const int ip = zinc(g, i), im = zdec(g, i);
      const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cjm = col_off(g, jm, i);
      const size_t cip = col_off(g, j, ip), cim = col_off(g, j, im);
      const size_t cjpip = col_off(g, jp, ip), cjpim = col_off(g, jp, im), cjmip = col_off(g, jm, ip);
      const double tc = temp[c + k];
      const double vxc = vx[c + k], vxp = vx[c + kp];
      const double vyc = vy[c + k], vyjp = vy[cjp + k];
      const double vzc = vz[c + k], vzip = vz[cip + k];
      const double vxm = 0.5 * (vxc + vxp), vym = 0.5 * (vyc + vyjp), vzm = 0.5 * (vzc + vzip);
      acc[0] += tc;
      acc[1] += vym;
      acc[2] += vzm;
      acc[3] += vxm * tc;
      acc[4] += vym * tc;
      acc[5] += vzm * tc;
      acc[6] += tc * tc;
      acc[7] += 0.5 * (vxc * vxc + vxp * vxp);
      acc[8] += 0.5 * (vyc * vyc + vyjp * vyjp);
      acc[9] += 0.5 * (vzc * vzc + vzip * vzip);
      acc[10] += 0.25 * (vxc + vxp) * (vyc + vyjp);
      acc[11] += 0.25 * (vxc + vxp) * (vzc + vzip);
      acc[12] += 0.25 * (vyc + vyjp) * (vzc + vzip);
      // chiT: horizontal gradients, then the wall-normal one with the plate values at the walls
      const double tz = (temp[cip + k] - temp[cim + k]) * 0.5 * g.dz;
      const double ty = (temp[cjp + k] - temp[cjm + k]) * 0.5 * g.dy;
      double tx;
      const size_t pl = (size_t)j + (size_t)g.nym * i;
      if (lo)
        tx = temp[c + 1] - tc + 2.0 * g.tfixs * (tc - __ldg(t.tempbp + pl));
      else if (hi)
        tx = tc - temp[c + km] + 2.0 * g.tfixn * (__ldg(t.temptp + pl) - tc);
      else
        tx = temp[c + kp] - temp[c + km];
      acc[13] += tz * tz + ty * ty + (tx * tdx) * (tx * tdx);
      // epsilon: the seven interior terms, then the wall-normal derivatives of vz and vy
      const double dz = g.dz, dy = g.dy;
      const double e1 = (vzip - vzc) * dz;
      const double a2 = vy[cjpip + k] - vy[cjpim + k], b2 = vy[cip + k] - vy[cim + k];
      const double a3 = vx[cip + kp] - vx[cim + kp], b3 = vx[cip + k] - vx[cim + k];
      const double a4 = vz[cjpip + k] - vz[cjmip + k], b4 = vz[cjp + k] - vz[cjm + k];
      const double e5 = (vyjp - vyc) * dy;
      const double a6 = vx[cjp + kp] - vx[cjm + kp], b6 = vx[cjp + k] - vx[cjm + k];
      const double e7 = (vxp - vxc) * udx3m;
      double eps = e1 * e1 + 0.125 * dz * dz * (a2 * a2 + b2 * b2) + 0.125 * dz * dz * (a3 * a3 + b3 * b3) +
                   0.125 * dy * dy * (a4 * a4 + b4 * b4) + e5 * e5 + 0.125 * dy * dy * (a6 * a6 + b6 * b6) + e7 * e7;
      double zxi, zxc, yxj, yxc;  // d/dx of vz at (j, i+1), (j, i) and vy at (j+1, i), (j, i)
      const double vzip0 = vz[cip + k], vyjp0 = vy[cjp + k];
      if (lo) {
        zxi = vz[cip + 1] - vzip0 + g.inslws * 2.0 * (vzip0 - 0.0);
        zxc = vz[c + 1] - vzc + g.inslws * 2.0 * (vzc - 0.0);
        yxj = vy[cjp + 1] - vyjp0 + g.inslws * 2.0 * (vyjp0 - g.xminusu);
        yxc = vy[c + 1] - vyc + g.inslws * 2.0 * (vyc - g.xminusu);
      } else if (hi) {
        zxi = vzip0 - vz[cip + km] + g.inslwn * 2.0 * (0.0 - vzip0);
        zxc = vzc - vz[c + km] + g.inslwn * 2.0 * (0.0 - vzc);
        yxj = vyjp0 - vy[cjp + km] + g.inslwn * 2.0 * (g.xplusu - vyjp0);
        yxc = vyc - vy[c + km] + g.inslwn * 2.0 * (g.xplusu - vyc);
      } else {
        zxi = vz[cip + kp] - vz[cip + km];
        zxc = vz[c + kp] - vz[c + km];
        yxj = vy[cjp + kp] - vy[cjp + km];
        yxc = vy[c + kp] - vy[c + km];
      }
      eps += tdx2 * (zxi * zxi + zxc * zxc) + tdx2 * (yxj * yxj + yxc * yxc);
      acc[14] += eps;
    }
  }
  if (k < nxm) {
#pragma unroll
    for (int q = 0; q < kNumProfiles; ++q) partial[((size_t)blockIdx.x * kNumProfiles + q) * nxm + k] = acc[q];
  }
}

__global__ void k_mean_reduce(const double *__restrict__ partial, int nblocks, int nxm, double *__restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // e = q*nxm + k
  if (e >= kNumProfiles * nxm) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * kNumProfiles * nxm + e];
  out[e] = s;
}

}  // namespace afid

using namespace afid;

namespace afid {

// Profiles of the columns [col0, col0 + ncols) into host out[15 * nxm], normalised by ny_nz
// (the number of y-z points averaged over) with the instance's ren / pect.
int ctx_mean_profiles(afid_ctx_t *ctx, int col0, int ncols, double ny_nz, double ren, double pect, double *out) {
  const Geom &g = ctx->L.g;
  const int nxm = g.nxm;
  const int nb = std::min(ncols, 148 * 4);
  const size_t need = (size_t)nb * kNumProfiles * nxm + (size_t)kNumProfiles * nxm;
  if (ctx->stats_elems < need) {
    if (ctx->stats_buf) cudaFree(ctx->stats_buf);
    ctx->stats_buf = nullptr;
    ctx->stats_elems = 0;
    if (cudaMalloc(&ctx->stats_buf, need * sizeof(double)) != cudaSuccess) return AFID_E_ALLOC;
    ctx->stats_elems = need;
  }
  double *partial = ctx->stats_buf, *sums = ctx->stats_buf + (size_t)nb * kNumProfiles * nxm;
  const int threads = (nxm + 31) / 32 * 32;
  k_mean_partial<<<nb, threads, 0, ctx->stream>>>(g, ctx->L.t, ctx->vx, ctx->vy, ctx->vz, ctx->temp, col0, ncols,
                                                  partial);
  k_mean_reduce<<<(kNumProfiles * nxm + 255) / 256, 256, 0, ctx->stream>>>(partial, nb, nxm, sums);
  ctx->launches += 2;
  cudaError_t e = cudaGetLastError();
  std::vector<double> h((size_t)kNumProfiles * nxm);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx_fail(ctx, e);
  // CalcMeanProfiles.F90:88-102 (x inym x inzm), square roots of the rms rows, :203-207
  const double inv = 1.0 / ny_nz;
  for (int q = 0; q < kNumProfiles; ++q)
    for (int k = 0; k < nxm; ++k) {
      double v = h[(size_t)q * nxm + k] * inv;
      if (q >= 6 && q <= 9) v = std::sqrt(v);
      if (q == 13) v /= pect;
      if (q == 14) v /= ren;
      out[(size_t)q * nxm + k] = v;
    }
  return AFID_OK;
}

}  // namespace afid

extern "C" int afid_gpu_mean_profiles(afid_ctx_t *ctx, double *out) {
  if (!ctx || !out || ctx->L.g.batch) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  return ctx_mean_profiles(ctx, 0, g.nym * g.nzm, (double)g.nym * (double)g.nzm, g.ren, g.pect, out);
}

// ------------------------------------------------------------------------------------------
// Spectra (spectra.F90): the y r2c + z c2c Fourier coefficients of vx, vy, vz and temp at
// k = 1..nxm, normalised by 1/(nym*nzm) (CalcFourierCoef, :70-96), accumulated as dt*|F|^2
// (AddRealSpectrum, :101-114) and divided by the averaging interval when read (WriteSpectra).
// The transforms are the Poisson solver's forward kernels with the field as their input.
// ------------------------------------------------------------------------------------------
namespace afid {

template <typename C>
__global__ void k_spec_acc(const C *__restrict__ spec, int nxm, int nyh, int nzm, int ldxc, double dt,
                           double *__restrict__ acc) {
  const size_t n = (size_t)nxm * nyh * nzm;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % nxm);
    const size_t m = e / nxm;  // ky + nyh*kz
    const C v = spec[m * ldxc + k];
    const double re = (double)v.x, im = (double)v.y;
    acc[e] += dt * (re * re + im * im);
  }
}

}  // namespace afid

extern "C" {

int afid_gpu_spectra_reset(afid_ctx_t *ctx) {
  if (!ctx || ctx->L.g.batch) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const size_t n = (size_t)4 * g.nxm * g.nyh * g.nzm;
  if (!ctx->spec_acc) {
    if (cudaMalloc(&ctx->spec_acc, n * sizeof(double)) != cudaSuccess) {
      ctx->spec_acc = nullptr;
      return AFID_E_ALLOC;
    }
  }
  ctx->spec_tav = 0.0;
  cudaError_t e = cudaMemsetAsync(ctx->spec_acc, 0, n * sizeof(double), ctx->stream);
  return e == cudaSuccess ? AFID_OK : ctx_fail(ctx, e);
}

int afid_gpu_spectra_update(afid_ctx_t *ctx, double dt) {
  if (!ctx || ctx->L.g.batch || !(dt > 0.0)) return AFID_E_INVALID;
  if (!ctx->spec_acc) {
    const int s = afid_gpu_spectra_reset(ctx);
    if (s != AFID_OK) return s;
  }
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const size_t n = (size_t)g.nxm * g.nyh * g.nzm;
  SubstepBuffers b = ctx_buffers(ctx);
  const double *fields[4] = {ctx->vx, ctx->vy, ctx->vz, ctx->temp};
  for (int f = 0; f < 4; ++f) {
    b.fft_field = fields[f];
    cudaError_t e = launch_stage(ctx->L, b, 0, Stage::DivFftY);
    if (e == cudaSuccess && g.nzm > 1) e = launch_stage(ctx->L, b, 0, Stage::FftZFwd);
    if (e != cudaSuccess) return ctx_fail(ctx, e);
    double *acc = ctx->spec_acc + (size_t)f * n;
    const int nb = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    if (ctx->L.mixed)
      k_spec_acc<<<nb, 256, 0, ctx->stream>>>((const float2 *)ctx->spec, g.nxm, g.nyh, g.nzm, g.ldxc, dt, acc);
    else
      k_spec_acc<<<nb, 256, 0, ctx->stream>>>((const double2 *)ctx->spec, g.nxm, g.nyh, g.nzm, g.ldxc, dt, acc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_fail(ctx, e);
    ctx->launches += (g.nzm > 1) ? 3 : 2;
  }
  ctx->spec_tav += dt;
  return AFID_OK;
}

int afid_gpu_spectra_read(afid_ctx_t *ctx, int which, double *out, double *tav) {
  if (!ctx || !out || which < 0 || which > 3 || !ctx->spec_acc || !(ctx->spec_tav > 0.0)) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const size_t n = (size_t)g.nxm * g.nyh * g.nzm;
  cudaError_t e = cudaMemcpyAsync(out, ctx->spec_acc + (size_t)which * n, n * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx_fail(ctx, e);
  const double inv = 1.0 / ctx->spec_tav;  // WriteSpectra: divide by the averaging interval
  for (size_t q = 0; q < n; ++q) out[q] *= inv;
  if (tav) *tav = ctx->spec_tav;
  return AFID_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Planes of a field (MakeMovie{X,Y,Z}Cut.F90): a wall-parallel plane at k gathered by a kernel,
// the others as strided 2-D copies.
// ------------------------------------------------------------------------------------------
namespace afid {

__global__ void k_xcut(const double *__restrict__ f, int ldx, int nym, int nzm, int k, double *__restrict__ out) {
  const size_t n = (size_t)nym * nzm;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = f[k + (size_t)ldx * e];
}

}  // namespace afid

extern "C" int afid_gpu_slice(afid_ctx_t *ctx, int which, int axis, int index, double *out) {
  if (!ctx || !out || which < 0 || which > 4 || ctx->L.g.batch) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const double *f = (which == 0) ? ctx->vx : (which == 1) ? ctx->vy : (which == 2) ? ctx->vz
                  : (which == 3) ? ctx->temp : ctx->pr;
  const size_t dp = (size_t)g.ldx * sizeof(double), w = (size_t)g.nx * sizeof(double);
  cudaError_t e = cudaSuccess;
  if (axis == 0) {  // x = const: out[i][j], nzm x nym
    if (index < 0 || index >= g.nx) return AFID_E_INVALID;
    const size_t n = (size_t)g.nym * g.nzm;
    if (ctx->stats_elems < n) {
      if (ctx->stats_buf) cudaFree(ctx->stats_buf);
      ctx->stats_buf = nullptr;
      ctx->stats_elems = 0;
      if (cudaMalloc(&ctx->stats_buf, n * sizeof(double)) != cudaSuccess) return AFID_E_ALLOC;
      ctx->stats_elems = n;
    }
    k_xcut<<<(int)std::min<size_t>((n + 255) / 256, 148 * 8), 256, 0, ctx->stream>>>(f, g.ldx, g.nym, g.nzm, index,
                                                                                      ctx->stats_buf);
    ctx->launches += 1;
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out, ctx->stats_buf, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  } else if (axis == 1) {  // y = const: out[i][k], nzm x nx
    if (index < 0 || index >= g.nym) return AFID_E_INVALID;
    e = cudaMemcpy2DAsync(out, w, f + (size_t)g.ldx * index, dp * g.nym, w, g.nzm, cudaMemcpyDeviceToHost, ctx->stream);
  } else if (axis == 2) {  // z = const: out[j][k], nym x nx
    if (index < 0 || index >= g.nzm) return AFID_E_INVALID;
    e = cudaMemcpy2DAsync(out, w, f + (size_t)g.ldx * g.nym * index, dp, w, g.nym, cudaMemcpyDeviceToHost, ctx->stream);
  } else {
    return AFID_E_INVALID;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? AFID_OK : ctx_fail(ctx, e);
}

// ---- plane means (h5tools/means.F90 ymean / zmean / ymeanr / zmeanr) ----------------------
// Mean over y (axis 1: out[i][k], planes x rows of nxc) or over z (axis 2: out[j][k]) of a
// field stored x-fastest with stride ld, ny rows per z-plane, nz planes.  The sum runs in the
// reference's order (the averaged index ascending) and is divided once at the end.
__global__ void k_plane_mean(const double *__restrict__ f, int ld, int ny, int nz, int nxc, int axis,
                             double *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;  // i (y-mean) or j (z-mean)
  if (k >= nxc) return;
  double acc = 0.0;
  if (axis == 1) {
    const double *p = f + (size_t)ld * ny * r + k;
    for (int j = 0; j < ny; ++j) acc += p[(size_t)ld * j];
    out[(size_t)r * nxc + k] = acc / (double)ny;
  } else {
    const double *p = f + (size_t)ld * r + k;
    for (int i = 0; i < nz; ++i) acc += p[(size_t)ld * ny * i];
    out[(size_t)r * nxc + k] = acc / (double)nz;
  }
}

namespace {
int plane_mean(afid_ctx_t *ctx, const double *f, int ld, int ny, int nz, int nxc, int axis, double *out) {
  const size_t n = (size_t)(axis == 1 ? nz : ny) * nxc;
  if (ctx->stats_elems < n) {
    if (ctx->stats_buf) cudaFree(ctx->stats_buf);
    ctx->stats_buf = nullptr;
    ctx->stats_elems = 0;
    if (cudaMalloc(&ctx->stats_buf, n * sizeof(double)) != cudaSuccess) return AFID_E_ALLOC;
    ctx->stats_elems = n;
  }
  const dim3 grid((unsigned)((nxc + 127) / 128), (unsigned)(axis == 1 ? nz : ny));
  k_plane_mean<<<grid, 128, 0, ctx->stream>>>(f, ld, ny, nz, nxc, axis, ctx->stats_buf);
  ctx->launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, ctx->stats_buf, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? AFID_OK : ctx_fail(ctx, e);
}
}  // namespace

extern "C" int afid_gpu_mean_plane(afid_ctx_t *ctx, int which, int axis, double *out) {
  if (!ctx || !out || which < 0 || which > 3 || (axis != 1 && axis != 2) || ctx->L.g.batch) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const double *f = (which == 0) ? ctx->vx : (which == 1) ? ctx->vy : (which == 2) ? ctx->vz : ctx->temp;
  return plane_mean(ctx, f, g.ldx, g.nym, g.nzm, g.nx, axis, out);
}

extern "C" int afid_gpu_sal_mean_plane(afid_ctx_t *ctx, int axis, double *out) {
  if (!ctx || !out || !ctx->sal || (axis != 1 && axis != 2)) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const SalGeom &sg = ctx->sal->sg;
  return plane_mean(ctx, ctx->sal->sal, sg.ldr, sg.nymr, sg.nzmr, sg.nxmr, axis, out);
}
