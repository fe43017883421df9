// afid_kernels.cu — sm_100a kernels of the RK3 flow + temperature substep.
//
// One substep (TimeMarcher.F90:38-133) is seven launches:
//   K1 k_explicit_implicit  ExplicitTerms{VX,VY,VZ,Temp} + ImplicitAndUpdate* + SolveImpEqnUpdate_*
//                           fused per x-column: one warp owns a (j,i) column, computes the four
//                           explicit terms and RHS, stores rux/ruy/ruz/rutemp and solves the four
//                           constant-matrix CN tridiagonals with a 32-chunk partition + PCR solve.
//   K2 k_div_fft_y          CalcLocalDivergence (pressure.F90:141-162) fused with the forward
//                           y r2c FFT (pressure.F90:174) and the 1/(nym*nzm) scaling (:179).
//   K3 k_fft_z<fwd>         forward z c2c FFT (pressure.F90:176).
//   K4 k_tridiag_pressure   SolveTridiagonalPressure (pressure.F90:201-236), warp per mode.
//   K5 k_fft_z<inv>         backward z c2c FFT (pressure.F90:189).
//   K6 k_ifft_y             backward y c2r FFT (pressure.F90:193) → phi.
//   K7 k_correct            RemoveDivergence + CorrectPressure (pressure.F90:240-301).
// plus k_cn_tables (once per step: CN factor tables for the three matrices and three substeps)
// and the reductions k_cfl / k_divmax / k_globals.
//
// Template parameter TE is the type of the explicit terms and of the stored RK3 history
// (double, or float for the mixed path); TS is the type of the spectral transforms.  The
// state (vx, vy, vz, temp, pr), the RHS assembly and every tridiagonal solve are FP64.
#include <algorithm>
#include <type_traits>

#include <cuda.h>

#include "afid_device.cuh"
#include "afid_internal.h"
#include "afid_k1.cuh"

namespace afid {

// ------------------------------------------------------------------------------------------
// CN tridiagonal factor tables.
//
// The matrices of SolveImpEqnUpdate_X.F90:27-42, SolveImpEqnUpdate_YZ.F90:25-36 and
// SolveImpEqnUpdate_Temp.F90:25-36 are identical for every (j,i) column: rows normalised by
// ackl_b = 1/(1 - ac*betadx), unit diagonal, a = -am*betadx*ackl_b, c = -ap*betadx*ackl_b.
// For vx the identity rows 1 and nx (whose RHS is zeroed, SolveImpEqnUpdate_X.F90:56-57) are
// eliminated, leaving rows k = 2..nxm.  Rows are split into 32 chunks of M (lane l owns rows
// l*M .. l*M+M-1, padded with identity rows); the first row of each chunk is an interface
// unknown.  Per lane the table holds the Thomas factors of the M-1 interior rows, their
// responses v/w to unit interface values, and the coefficients of the 32-unknown reduced
// system in PCR form.  Layout (doubles): [sc 32M][a 32M][inv 32M][cp 32M][v 32M][w 32M]
// [as 32][cs 32][rinvB 32][pa 5x32][pg 5x32][pn 5x32], interior arrays as [q][lane].
// ------------------------------------------------------------------------------------------

struct CnMatrixDesc {
  const double *am, *ac, *ap;
  int off, n;          // first reference row (0-based) and number of unknowns
  int temperature;     // betadx = 0.5*al*dt/pect instead of beta*al
};

struct CnBuildArgs {
  CnMatrixDesc mat[3];
  double al[3], ga[3], ro[3];
  double dt, beta, pect, ren;
  int ns0, nsub;       // substeps ns0 .. ns0+nsub-1 are built
  int nmat;            // matrices per substep (tables at (slot * nmat + m))
  // batch mode: one table set per instance, dt from dt_dev[instance] (beta = dt/ren/2),
  // ren/pect from inst[instance]; idle instances are skipped
  const double *dt_dev;
  const InstScal *inst;
  const unsigned char *active;
};

__global__ void k_cn_tables(CnBuildArgs args, int M, double *__restrict__ tab,
                            StepCoef *__restrict__ sc) {
  const int lane = threadIdx.x;
  const int m = blockIdx.x % args.nmat;
  const int sub = (blockIdx.x / args.nmat) % args.nsub;
  const int b = blockIdx.x / (args.nmat * args.nsub);  // instance (batch mode), else 0
  const int ns = args.ns0 + sub;
  const double al = args.al[sub];
  double dt = args.dt, beta = args.beta, ren = args.ren, pect = args.pect;
  int slot = ns;
  if (args.dt_dev) {
    if (args.active && !args.active[b]) return;
    dt = args.dt_dev[b];
    ren = args.inst[b].ren;
    pect = args.inst[b].pect;
    beta = dt / ren * 0.5;  // TimeMarcher.F90:28
    slot = 3 * b + ns;
  }
  if (m == 0 && lane == 0) {
    StepCoef c;
    c.al = al;
    c.ga = args.ga[sub];
    c.ro = args.ro[sub];
    c.dt = dt;
    c.beta = beta;
    c.alre = al / ren;
    c.alpec = al / pect;
    sc[slot] = c;
  }
  const CnMatrixDesc d = args.mat[m];
  const double betadx = d.temperature ? 0.5 * al * dt / pect : beta * al;
  double *T = tab + (size_t)(slot * args.nmat + m) * cn_table_size(M);
  double *Tsc = T, *Ta = T + 32 * M, *Tinv = T + 64 * M, *Tcp = T + 96 * M, *Tv = T + 128 * M,
         *Tw = T + 160 * M, *Tl = T + 192 * M;
  const int n = d.n;
  auto coef = [&](int r, double &a, double &c, double &s) {
    if (r >= n) { a = 0.0; c = 0.0; s = 0.0; return; }
    const int k = r + d.off;
    const double ackl_b = 1.0 / (1.0 - d.ac[k] * betadx);
    a = (r == 0) ? 0.0 : -d.am[k] * betadx * ackl_b;
    c = (r == n - 1) ? 0.0 : -d.ap[k] * betadx * ackl_b;
    s = ackl_b;
  };
  const int s0 = lane * M;
  double as_, cs_, scl;
  coef(s0, as_, cs_, scl);
  Tsc[s0] = scl;
  double cp_prev = 0.0, v_prev = 0.0;
  for (int q = 1; q < M; ++q) {
    double a, c, s;
    coef(s0 + q, a, c, s);
    Tsc[s0 + q] = s;
    const double den = (q > 1) ? 1.0 - a * cp_prev : 1.0;
    const double inv = 1.0 / den;
    const double cp = c * inv;
    const double vp = ((q == 1) ? -a : -a * v_prev) * inv;
    const double wp = (q == M - 1) ? -c * inv : 0.0;
    Ta[q * 32 + lane] = a;
    Tinv[q * 32 + lane] = inv;
    Tcp[q * 32 + lane] = cp;
    Tv[q * 32 + lane] = vp;
    Tw[q * 32 + lane] = wp;
    cp_prev = cp;
    v_prev = vp;
  }
  for (int q = M - 2; q >= 1; --q) {
    Tv[q * 32 + lane] -= Tcp[q * 32 + lane] * Tv[(q + 1) * 32 + lane];
    Tw[q * 32 + lane] -= Tcp[q * 32 + lane] * Tw[(q + 1) * 32 + lane];
  }
  double A, B, C;
  if (M == 1) {
    A = as_;
    B = 1.0;
    C = cs_;
  } else {
    double vl = __shfl_up_sync(0xffffffffu, Tv[(M - 1) * 32 + lane], 1);
    double wl = __shfl_up_sync(0xffffffffu, Tw[(M - 1) * 32 + lane], 1);
    if (lane == 0) { vl = 0.0; wl = 0.0; }
    A = as_ * vl;
    B = 1.0 + as_ * wl + cs_ * Tv[32 + lane];
    C = (lane == 31) ? 0.0 : cs_ * Tw[32 + lane];
  }
  const double rinvB = 1.0 / B;
  Tl[lane] = as_;
  Tl[32 + lane] = cs_;
  Tl[64 + lane] = rinvB;
  double al_ = A * rinvB, ga_ = C * rinvB;
  for (int lev = 0, h = 1; lev < 5; ++lev, h <<= 1) {
    double am = __shfl_up_sync(0xffffffffu, al_, h);
    double gm = __shfl_up_sync(0xffffffffu, ga_, h);
    double ap = __shfl_down_sync(0xffffffffu, al_, h);
    double gp = __shfl_down_sync(0xffffffffu, ga_, h);
    if (lane < h) { am = 0.0; gm = 0.0; }
    if (lane + h >= 32) { ap = 0.0; gp = 0.0; }
    const double nrm = 1.0 / (1.0 - al_ * gm - ga_ * ap);
    Tl[96 + lev * 32 + lane] = al_;
    Tl[256 + lev * 32 + lane] = ga_;
    Tl[416 + lev * 32 + lane] = nrm;
    const double na = -al_ * am * nrm, ng = -ga_ * gp * nrm;
    al_ = na;
    ga_ = ng;
  }
}

// K1 (explicit terms + RHS + CN solves) lives in afid_k1.cuh.

// ------------------------------------------------------------------------------------------
// K2: divergence (pressure.F90:147-158) fused with the forward y r2c FFT (pressure.F90:174)
// and the 1/(nym*nzm) normalisation (pressure.F90:179).  Block = (x tile of TX points, z
// index i).  Pairs of x points are packed as one complex sequence (re, im), transformed, and
// split with X_k = (Z_k + conj Z_{N-k})/2, Y_k = (Z_k - conj Z_{N-k})/(2i).
// ------------------------------------------------------------------------------------------
template <int TX, typename TS>
__global__ void __launch_bounds__(256)
    k_div_fft_y(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
                const double *__restrict__ vx, const double *__restrict__ vy,
                const double *__restrict__ vz, typename Cplx<TS>::type *__restrict__ spec,
                FftPlan pl, const typename Cplx<TS>::type *__restrict__ tw, const double *__restrict__ field) {
  using C = typename Cplx<TS>::type;
  extern __shared__ __align__(16) unsigned char smem_raw_k2[];
  C *b0 = reinterpret_cast<C *>(smem_raw_k2);
  const int k0 = blockIdx.x * TX, i = blockIdx.y;
  Geom g = g0;
  const int N = g.nym, B = TX / 2;
  C *b1 = b0 + (size_t)B * N;
  if (!inst_active(g, i)) return;
  bind_instance(g, i);
  const int ip = zinc(g, i);
  const StepCoef sc = sc_all[sc_slot(g, i, ns)];
  const double usdtal = 1.0 / (sc.dt * sc.al);
  const int tx = threadIdx.x % TX;
  const int k = k0 + tx;
#pragma unroll 4
  for (int j = threadIdx.x / TX; j < N; j += blockDim.x / TX) {
    double dv = 0.0;
    if (k < g.nxm && field) {
      dv = __ldg(field + col_off(g, j, i) + k);
    } else if (k < g.nxm) {
      const int jp = wrap_inc(j, N);
      const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cip = col_off(g, j, ip);
      const double dqcap = (__ldg(vz + cip + k) - __ldg(vz + c + k)) * g.dz +
                           (__ldg(vy + cjp + k) - __ldg(vy + c + k)) * g.dy +
                           (__ldg(vx + c + k + 1) - __ldg(vx + c + k)) * __ldg(t.udx3m + k);
      dv = dqcap * usdtal;
    }
    TS *d = reinterpret_cast<TS *>(&b0[(size_t)(tx >> 1) * N + j]);
    d[tx & 1] = (TS)dv;
  }
  __syncthreads();
  C *res = fft_block<false, TS>(b0, b1, B, pl, tw);
  const TS norm = (TS)(1.0 / (nz_norm(g) * (double)g.nym));
  const TS half = (TS)0.5;
  for (int e = threadIdx.x; e < g.nyh * TX; e += blockDim.x) {
    const int ex = e % TX, ky = e / TX;
    const int kk = k0 + ex;
    if (kk >= g.nxm) continue;
    const int p = ex >> 1;
    const C zk = res[(size_t)p * N + ky];
    const C zn = res[(size_t)p * N + (ky == 0 ? 0 : N - ky)];
    C X;
    if ((ex & 1) == 0) {
      X.x = (zk.x + zn.x) * half;
      X.y = (zk.y - zn.y) * half;
    } else {
      X.x = (zk.y + zn.y) * half;
      X.y = (zn.x - zk.x) * half;
    }
    X.x *= norm;
    X.y *= norm;
    spec[(size_t)(ky + (size_t)g.nyh * i) * g.ldxc + kk] = X;
  }
}

// K3 / K5: z c2c FFT in place on the spectrum.  Block = (x tile of TXZ points, ky).
template <int TXZ, bool INV, typename TS>
__global__ void __launch_bounds__(256)
    k_fft_z(Geom g, typename Cplx<TS>::type *__restrict__ spec, FftPlan pl,
            const typename Cplx<TS>::type *__restrict__ tw) {
  using C = typename Cplx<TS>::type;
  extern __shared__ __align__(16) unsigned char smem_raw_k3[];
  C *b0 = reinterpret_cast<C *>(smem_raw_k3);
  const int N = g.nzm;
  C *b1 = b0 + (size_t)TXZ * N;
  const int k0 = blockIdx.x * TXZ, ky = blockIdx.y;
  const size_t zstride = (size_t)g.nyh * g.ldxc;
  C *base = spec + (size_t)ky * g.ldxc + k0;
#pragma unroll 8
  for (int e = threadIdx.x; e < N * TXZ; e += blockDim.x) {
    const int ex = e % TXZ, iz = e / TXZ;
    C v;
    v.x = 0;
    v.y = 0;
    if (k0 + ex < g.nxm) v = base[(size_t)iz * zstride + ex];
    b0[(size_t)ex * N + iz] = v;
  }
  __syncthreads();
  C *res = fft_block<INV, TS>(b0, b1, TXZ, pl, tw);
  for (int e = threadIdx.x; e < N * TXZ; e += blockDim.x) {
    const int ex = e % TXZ, iz = e / TXZ;
    if (k0 + ex < g.nxm) base[(size_t)iz * zstride + ex] = res[(size_t)ex * N + iz];
  }
}

// ------------------------------------------------------------------------------------------
// K4: per (ky, kz) mode, the complex tridiagonal of pressure.F90:209-232.  The reference scales
// row k by 1/(acphk(k)-ak2(j)-ak1(i)) and puts 1+1e-15 on the diagonal; the same system is
// solved here unscaled (amphk, (acphk-ak2-ak1)(1+1e-15), apphk), which saves a reciprocal per
// row.  One warp per mode; rows are split into 32 chunks of M (partition + PCR as in the CN
// solve, with factors computed per mode).  The (0,0) mode is singular up to
// the 1e-15 shift (the reference lets LAPACK return an arbitrary constant); here its last
// equation is replaced by phi = 0, which fixes that constant without changing gradients.
// A zero pivot sets AFID_E_SINGULAR (the reference aborts, pressure.F90:225-229).
// ------------------------------------------------------------------------------------------
template <int M, int WPB, typename TS>
__global__ void __launch_bounds__(WPB * 32)
    k_tridiag_pressure(Geom g, Tables t, typename Cplx<TS>::type *__restrict__ spec,
                       int *__restrict__ err) {
  using C = typename Cplx<TS>::type;
  extern __shared__ double smem_k4[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sys = blockIdx.x * WPB + warp;
  if (sys >= g.nyh * g.nzm) return;
  const int ky = sys % g.nyh, kz = sys / g.nyh;
  if (!inst_active(g, kz)) return;  // whole warp (batch mode: kz numbers the instance)
  // the singular (0,0) mode; in batch mode every instance's ky = 0 mode (nzm = 1 each)
  const bool pin = (ky == 0 && (kz == 0 || g.batch));
  constexpr int LD = chunk_ld(M);
  // M <= 8: the diagonal is kept in shared memory too (a fifth array costs no resident block)
  constexpr bool kStoreB = (M <= 8);
  constexpr int NA = kStoreB ? 5 : 4;
  double *sa = smem_k4 + warp * (NA * LD * M);
  double *sc_ = sa + LD * M, *sdr = sa + 2 * LD * M, *sdi = sa + 3 * LD * M, *sb = sa + 4 * LD * M;
  C *colp = spec + (size_t)sys * g.ldxc;
  const int n = g.nxm;
  const double akj = __ldg(t.ak2 + (g.batch ? (size_t)kz * g.nym : 0) + ky);
  const double aki = g.batch ? 0.0 : __ldg(t.ak1 + kz);
#pragma unroll
  for (int tt = 0; tt < M; ++tt) {
    const int r = lane + 32 * tt;
    const int s = (r % M) * LD + r / M;
    // the rows unnormalised: the reference's row scaling 1/(acphk - ak2 - ak1) with unit-plus-
    // 1e-15 diagonal is the same system as diagonal (acphk - ak2 - ak1)(1 + 1e-15)
    double a = 0.0, c = 0.0, dr = 0.0, di = 0.0, b = 1.0;
    if (r < n) {
      a = (r > 0) ? __ldg(t.amphk + r) : 0.0;
      c = (r < n - 1) ? __ldg(t.apphk + r) : 0.0;
      if (kStoreB) b = (__ldg(t.acphk + r) - akj - aki) * (1.0 + 1.0e-15);
      const C v = colp[r];
      dr = (double)v.x;
      di = (double)v.y;
      if (pin && r == n - 1) { a = 0.0; dr = 0.0; di = 0.0; b = 1.0; }
    }
    sa[s] = a;
    sc_[s] = c;
    sdr[s] = dr;
    sdi[s] = di;
    if (kStoreB) sb[s] = b;
  }
  __syncwarp();
  const int s0 = lane * M;
  // diagonal of row s0 + q (identity for padding rows and the pinned row)
  auto diag = [&](int q) -> double {
    if constexpr (kStoreB) return sb[q * LD + lane];
    const int r = s0 + q;
    return (r < n && !(pin && r == n - 1)) ? (__ldg(t.acphk + r) - akj - aki) * (1.0 + 1.0e-15) : 1.0;
  };
  double cp[M], yr[M], yi[M], v[M], w[M];
  bool bad = false;
  cp[0] = 0.0; yr[0] = 0.0; yi[0] = 0.0; v[0] = 0.0; w[0] = 0.0;
#pragma unroll
  for (int q = 1; q < M; ++q) {
    const double a = sa[q * LD + lane], c = sc_[q * LD + lane];
    const double den = (q > 1) ? diag(q) - a * cp[q - 1] : diag(q);
    bad |= (den == 0.0);
    const double inv = 1.0 / den;
    cp[q] = c * inv;
    const double dr = sdr[q * LD + lane], di = sdi[q * LD + lane];
    if (q > 1) {
      yr[q] = (dr - a * yr[q - 1]) * inv;
      yi[q] = (di - a * yi[q - 1]) * inv;
      v[q] = -a * v[q - 1] * inv;
    } else {
      yr[q] = dr * inv;
      yi[q] = di * inv;
      v[q] = -a * inv;
    }
    w[q] = (q == M - 1) ? -c * inv : 0.0;
  }
#pragma unroll
  for (int q = M - 2; q >= 1; --q) {
    yr[q] -= cp[q] * yr[q + 1];
    yi[q] -= cp[q] * yi[q + 1];
    v[q] -= cp[q] * v[q + 1];
    w[q] -= cp[q] * w[q + 1];
  }
  const double as_ = sa[lane], cs_ = sc_[lane];
  double A, B, Cc, Dr, Di;
  if constexpr (M == 1) {
    A = as_;
    B = diag(0);
    Cc = cs_;
    Dr = sdr[lane];
    Di = sdi[lane];
  } else {
    double vl = __shfl_up_sync(0xffffffffu, v[M - 1], 1);
    double wl = __shfl_up_sync(0xffffffffu, w[M - 1], 1);
    double yl_r = __shfl_up_sync(0xffffffffu, yr[M - 1], 1);
    double yl_i = __shfl_up_sync(0xffffffffu, yi[M - 1], 1);
    if (lane == 0) { vl = 0.0; wl = 0.0; yl_r = 0.0; yl_i = 0.0; }
    A = as_ * vl;
    B = diag(0) + as_ * wl + cs_ * v[1];
    Cc = (lane == 31) ? 0.0 : cs_ * w[1];
    Dr = sdr[lane] - as_ * yl_r - cs_ * yr[1];
    Di = sdi[lane] - as_ * yl_i - cs_ * yi[1];
  }
  bad |= (B == 0.0);
  const double rB = 1.0 / B;
  double al_ = A * rB, ga_ = Cc * rB, er = Dr * rB, ei = Di * rB;
#pragma unroll
  for (int h = 1; h < 32; h <<= 1) {
    double am = __shfl_up_sync(0xffffffffu, al_, h), gm = __shfl_up_sync(0xffffffffu, ga_, h);
    double ap = __shfl_down_sync(0xffffffffu, al_, h), gp = __shfl_down_sync(0xffffffffu, ga_, h);
    double erm = __shfl_up_sync(0xffffffffu, er, h), eim = __shfl_up_sync(0xffffffffu, ei, h);
    double erp = __shfl_down_sync(0xffffffffu, er, h), eip = __shfl_down_sync(0xffffffffu, ei, h);
    if (lane < h) { am = 0.0; gm = 0.0; erm = 0.0; eim = 0.0; }
    if (lane + h >= 32) { ap = 0.0; gp = 0.0; erp = 0.0; eip = 0.0; }
    const double dd = 1.0 - al_ * gm - ga_ * ap;
    bad |= (dd == 0.0);
    const double nrm = 1.0 / dd;
    er = (er - al_ * erm - ga_ * erp) * nrm;
    ei = (ei - al_ * eim - ga_ * eip) * nrm;
    const double na = -al_ * am * nrm, ng = -ga_ * gp * nrm;
    al_ = na;
    ga_ = ng;
  }
  double xnr = __shfl_down_sync(0xffffffffu, er, 1), xni = __shfl_down_sync(0xffffffffu, ei, 1);
  if (lane == 31) { xnr = 0.0; xni = 0.0; }
  sdr[lane] = er;
  sdi[lane] = ei;
#pragma unroll
  for (int q = 1; q < M; ++q) {
    sdr[q * LD + lane] = yr[q] + v[q] * er + w[q] * xnr;
    sdi[q * LD + lane] = yi[q] + v[q] * ei + w[q] * xni;
  }
  if (bad) atomicOr(err, 1);
  __syncwarp();
#pragma unroll 1
  for (int tt = 0; tt < M; ++tt) {
    const int r = lane + 32 * tt;
    if (r < n) {
      const int s = (r % M) * LD + r / M;
      C o;
      o.x = (TS)sdr[s];
      o.y = (TS)sdi[s];
      colp[r] = o;
    }
  }
}

// K6: backward y c2r FFT (pressure.F90:193), unnormalised.  The half spectrum of two x
// points is extended Hermitian-symmetrically (imaginary parts of the DC and Nyquist bins are
// ignored, as a c2r transform does), packed as Z = X + iY, transformed, and split into
// Re -> phi(k0), Im -> phi(k0+1).
template <int TX, typename TS>
__global__ void __launch_bounds__(256)
    k_ifft_y(Geom g, const typename Cplx<TS>::type *__restrict__ spec, TS *__restrict__ phi,
             FftPlan pl, const typename Cplx<TS>::type *__restrict__ tw) {
  using C = typename Cplx<TS>::type;
  extern __shared__ __align__(16) unsigned char smem_raw_k6[];
  C *b0 = reinterpret_cast<C *>(smem_raw_k6);
  const int N = g.nym, B = TX / 2;
  C *b1 = b0 + (size_t)B * N;
  const int k0 = blockIdx.x * TX, i = blockIdx.y;
  if (!inst_active(g, i)) return;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * B; e += blockDim.x) {
    const int p = e % B, j = e / B;
    const bool cj = (2 * j > N);
    const int jj = cj ? N - j : j;
    const int ka = k0 + 2 * p, kb = ka + 1;
    const C *src = spec + (size_t)(jj + (size_t)g.nyh * i) * g.ldxc;
    C X, Y;
    X.x = 0; X.y = 0; Y.x = 0; Y.y = 0;
    if (ka < g.nxm) X = src[ka];
    if (kb < g.nxm) Y = src[kb];
    if (cj) { X.y = -X.y; Y.y = -Y.y; }
    if (jj == 0 || 2 * jj == N) { X.y = 0; Y.y = 0; }
    C Z;
    Z.x = X.x - Y.y;
    Z.y = X.y + Y.x;
    b0[(size_t)p * N + j] = Z;
  }
  __syncthreads();
  const C *res = fft_block<true, TS>(b0, b1, B, pl, tw);
  for (int e = threadIdx.x; e < N * TX; e += blockDim.x) {
    const int ex = e % TX, j = e / TX;
    const int k = k0 + ex;
    if (k >= g.nxm) continue;
    const C z = res[(size_t)(ex >> 1) * N + j];
    phi[col_off(g, j, i) + k] = (ex & 1) ? z.y : z.x;
  }
}

// K7: RemoveDivergence (pressure.F90:245-266) out of place (intermediate velocities -> state)
// and CorrectPressure (pressure.F90:276-300) in place.  Thread per (k, j, i).
__device__ __forceinline__ double2 make_v2(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 make_v2(float a, float b) { return make_float2(a, b); }

template <typename TS>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// K7: RemoveDivergence (pressure.F90:240-267) + CorrectPressure (pressure.F90:270-301).  Each
// thread updates the two x-neighbours k0 = 2*tx and k0+1 with 16-byte (8-byte for FP32 phi)
// vector loads and stores; the x-neighbours of the pair come from the adjacent threads.
template <typename TS>
__global__ void __launch_bounds__(256)
    k_correct(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
              const double *__restrict__ vxh, const double *__restrict__ vyh,
              const double *__restrict__ vzh, double *__restrict__ vx, double *__restrict__ vy,
              double *__restrict__ vz, double *__restrict__ pr, const TS *__restrict__ phi) {
  using V = typename Vec2<TS>::type;
  const int k0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  Geom g = g0;
  // threads past the end of the row still take part in the neighbour exchange below
  const bool row_ok = (j < g.nym) && inst_active(g, i);
  if (!row_ok) return;  // whole warps share j (blockDim.x is a multiple of 32)
  bind_instance(g, i);
  const int nxm = g.nxm;
  const bool in0 = k0 < nxm, in1 = k0 + 1 < nxm;
  const StepCoef sc = sc_all[sc_slot(g, i, ns)];
  const int jm = wrap_dec(j, g.nym), jp = wrap_inc(j, g.nym);
  const int im = zdec(g, i), ip = zinc(g, i);
  const size_t c = col_off(g, j, i);
  // pairs (k0, k0+1): k0 even and every column starts on a multiple of 8 elements
  V ph2 = make_v2(TS(0), TS(0)), pjm2 = ph2, pjp2 = ph2, pim2 = ph2, pip2 = ph2;
  double2 uxh = make_double2(0.0, 0.0), uyh = uxh, uzh = uxh, upr = uxh;
  if (in0) {
    ph2 = *reinterpret_cast<const V *>(phi + c + k0);
    pjm2 = *reinterpret_cast<const V *>(phi + col_off(g, jm, i) + k0);
    pjp2 = *reinterpret_cast<const V *>(phi + col_off(g, jp, i) + k0);
    pim2 = *reinterpret_cast<const V *>(phi + col_off(g, j, im) + k0);
    pip2 = *reinterpret_cast<const V *>(phi + col_off(g, j, ip) + k0);
    uxh = __ldg(reinterpret_cast<const double2 *>(vxh + c + k0));
    uyh = __ldg(reinterpret_cast<const double2 *>(vyh + c + k0));
    uzh = __ldg(reinterpret_cast<const double2 *>(vzh + c + k0));
    upr = *reinterpret_cast<const double2 *>(pr + c + k0);
  }
  // x-neighbours: phi(k0-1) is the left thread's second value, phi(k0+2) the right thread's
  // first; the lanes at the ends of a warp load theirs
  const int lane = threadIdx.x & 31;
  double left = __shfl_up_sync(0xffffffffu, (double)ph2.y, 1);
  double right = __shfl_down_sync(0xffffffffu, (double)ph2.x, 1);
  if (!in0) return;
  if (lane == 0) left = (k0 > 0) ? (double)phi[c + k0 - 1] : 0.0;
  if (lane == 31 || k0 + 2 >= nxm) right = (k0 + 2 < nxm) ? (double)phi[c + k0 + 2] : 0.0;
  const double ph0 = (double)ph2.x, ph1 = (double)ph2.y;
  const double phkm0 = (k0 == 0) ? ph0 : left;           // kmv(1) = 1
  const double phkp1 = (k0 + 1 == nxm - 1) ? ph1 : right;  // kpv(nxm) = nxm
  const double aldt = sc.al * sc.dt;
  const double udy = aldt * g.dy, udz = aldt * g.dz;
  const double be = sc.al * sc.beta;
  const double2 ud = __ldg(reinterpret_cast<const double2 *>(t.udx3c + k0));
  const double2 am = __ldg(reinterpret_cast<const double2 *>(t.amphk + k0));
  const double2 ac = __ldg(reinterpret_cast<const double2 *>(t.acphk + k0));
  const double2 ap = __ldg(reinterpret_cast<const double2 *>(t.apphk + k0));
  double2 ox, oy, oz, op;
  // cell k0
  ox.x = uxh.x - (ph0 - phkm0) * (aldt * ud.x);
  oy.x = uyh.x - (ph0 - (double)pjm2.x) * udy;
  oz.x = uzh.x - (ph0 - (double)pim2.x) * udz;
  op.x = upr.x + ph0 -
         be * (((double)pip2.x - 2.0 * ph0 + (double)pim2.x) * g.dzq +
               ((double)pjp2.x - 2.0 * ph0 + (double)pjm2.x) * g.dyq + ((in1 ? ph1 : ph0) * ap.x + ph0 * ac.x + phkm0 * am.x));
  if (in1) {
    ox.y = uxh.y - (ph1 - ph0) * (aldt * ud.y);
    oy.y = uyh.y - (ph1 - (double)pjm2.y) * udy;
    oz.y = uzh.y - (ph1 - (double)pim2.y) * udz;
    op.y = upr.y + ph1 -
           be * (((double)pip2.y - 2.0 * ph1 + (double)pim2.y) * g.dzq +
                 ((double)pjp2.y - 2.0 * ph1 + (double)pjm2.y) * g.dyq + (phkp1 * ap.y + ph1 * ac.y + ph0 * am.y));
    *reinterpret_cast<double2 *>(vx + c + k0) = ox;
    *reinterpret_cast<double2 *>(vy + c + k0) = oy;
    *reinterpret_cast<double2 *>(vz + c + k0) = oz;
    *reinterpret_cast<double2 *>(pr + c + k0) = op;
  } else {
    vx[c + k0] = ox.x;
    vy[c + k0] = oy.x;
    vz[c + k0] = oz.x;
    pr[c + k0] = op.x;
  }
  if (k0 + 1 >= nxm - 1) vx[c + nxm] = __ldg(vxh + c + nxm);  // the upper wall value is copied
}

// ------------------------------------------------------------------------------------------
// Reductions.  Maxima of non-negative doubles are combined with atomicMax on their bit
// patterns (order-preserving for x >= 0), so the result does not depend on block order.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <bool DIV>
__global__ void __launch_bounds__(256)
    k_max_reduce(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                 const double *__restrict__ vz, unsigned long long *__restrict__ out) {
  __shared__ double red[8];
  double m = 0.0;
  const int lane = threadIdx.x & 31;
  const int ncol = g.nym * g.nzm;
  const int wstride = gridDim.x * (blockDim.x >> 5);
  for (int cidx = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); cidx < ncol; cidx += wstride) {
    const int j = cidx % g.nym, i = cidx / g.nym;
    const int jp = wrap_inc(j, g.nym), ip = zinc(g, i);
    const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cip = col_off(g, j, ip);
    for (int k = lane; k < g.nxm; k += 32) {
      double q;
      if (DIV) {  // CheckDivergence.F90:36-39
        const double dq = (vz[cip + k] - vz[c + k]) * g.dz + (vy[cjp + k] - vy[c + k]) * g.dy +
                          (vx[c + k + 1] - vx[c + k]) * t.udx3m[k];
        q = fabs(dq);
      } else {  // CalcMaxCFL.F90:36-40
        q = fabs((vz[c + k] + vz[cip + k]) * 0.5 * g.dz) + fabs((vy[c + k] + vy[cjp + k]) * 0.5 * g.dy) +
            fabs((vx[c + k] + vx[c + k + 1]) * 0.5 * t.udx3m[k]);
      }
      m = nan_max(m, q);
    }
  }
  m = warp_max(m);
  if (lane == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    v = warp_max(v);
    if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
  }
}

// Volume sums of GlobalQuantities.F90:39-60 per block, written to partial[block*3 + {0,1,2}]
// (T*vx_centre*g3rc, (vx^2+vy^2+vz^2)*g3rc, T*g3rc) and summed in fixed order afterwards.
__global__ void __launch_bounds__(256)
    k_globals_partial(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                      const double *__restrict__ vz, const double *__restrict__ temp,
                      double *__restrict__ partial) {
  __shared__ double red[3][8];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  const int lane = threadIdx.x & 31;
  const int ncol = g.nym * g.nzm;
  const int wstride = gridDim.x * (blockDim.x >> 5);
  for (int cidx = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); cidx < ncol; cidx += wstride) {
    const size_t c = (size_t)cidx * g.ldx;
    for (int k = lane; k < g.nxm; k += 32) {
      const double fac2 = t.g3rc[k];
      const double vxcen = (vx[c + k] + vx[c + k + 1]) * 0.5;
      const double tc = temp[c + k];
      s0 += tc * vxcen * fac2;
      s1 += fac2 * (vz[c + k] * vz[c + k] + vy[c + k] * vy[c + k] + vx[c + k] * vx[c + k]);
      s2 += tc * fac2;
    }
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (lane == 0) {
    red[0][threadIdx.x >> 5] = s0;
    red[1][threadIdx.x >> 5] = s1;
    red[2][threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    partial[blockIdx.x * 3 + threadIdx.x] = v;
  }
}

__global__ void k_sum_partials(const double *__restrict__ partial, int nblocks, double *__restrict__ out) {
  __shared__ double red[3][8];
  double s[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < 3; ++q) s[q] += partial[b * 3 + q];
  for (int q = 0; q < 3; ++q) {
    s[q] = warp_sum(s[q]);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = s[q];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    out[threadIdx.x] = v;
  }
}

// ------------------------------------------------------------------------------------------
// Warp-FFT variants of K2, K3/K5, K6 (N = 32*N1).  Shared memory only transposes between the
// coalesced HBM layout and the per-warp sequences (each warp owns one sequence); after the
// transform lane l, register k1 holds element k1 + N1*bitrev5(l).
// ------------------------------------------------------------------------------------------
// Column swizzle of the z-transform tile [row][8 x points] (16-byte elements): element (r, w)
// sits at r*8 + (w ^ zsw(r)).  Keeps the coalesced row accesses, the per-warp column reads and
// the bit-reversed per-warp writes at most 2-way bank conflicted for every supported N1.
__device__ __forceinline__ int zsw(int r) { return (r ^ (r >> 2) ^ (r >> 6)) & 7; }

// Tile of 8 complex columns per row, swizzled: element (r, c) at r*8 + (c ^ zsw(r)).
__device__ __forceinline__ int tsw(int r, int c) { return r * 8 + (c ^ zsw(r)); }

// K2w: divergence + forward y r2c.  Block: 16 x points = 8 pairs (8 warps, one pair per warp)
// at one z index i.  The real tile is the complex tile read as (re, im) = (x point 2c, 2c+1).
template <int N1, typename TS>
__global__ void __launch_bounds__(256)
    k_div_fft_y_w(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
                  const double *__restrict__ vx, const double *__restrict__ vy,
                  const double *__restrict__ vz, typename Cplx<TS>::type *__restrict__ spec,
                  const typename Cplx<TS>::type *__restrict__ tw, const double *__restrict__ field) {
  using C = typename Cplx<TS>::type;
  constexpr int N = 32 * N1;
  extern __shared__ __align__(16) unsigned char smem_k2w[];
  C *T = reinterpret_cast<C *>(smem_k2w);  // [N][8] swizzled
  TS *Tr = reinterpret_cast<TS *>(smem_k2w);
  constexpr bool LT = lane_table_fits((size_t)N * 8 * sizeof(C), lane_table_bytes<N1, C>());
  C *stw = T + N * 8;  // lane twiddles (when LT)
  const int k0 = blockIdx.x * 16, i = blockIdx.y;
  Geom g = g0;
  if (!inst_active(g, i)) return;
  if constexpr (LT) fill_lane_twiddles<TS, N1>(stw, tw);
  bind_instance(g, i);
  const int ip = zinc(g, i);
  const StepCoef sc = sc_all[sc_slot(g, i, ns)];
  const double usdtal = 1.0 / (sc.dt * sc.al);
  // thread pair q holds the x points (kk, kk+1) = (k0 + 2q, k0 + 2q + 1), loaded with 16-byte
  // vector loads, and stores them as the packed complex column q
  const int q = threadIdx.x & 7, kk = k0 + 2 * q;
  const int nxm = g.nxm;
  const double2 ux = (kk < nxm) ? __ldg(reinterpret_cast<const double2 *>(t.udx3m + kk)) : make_double2(0.0, 0.0);
  (void)Tr;
#pragma unroll 4
  for (int j = threadIdx.x >> 3; j < N; j += 32) {
    double dv0 = 0.0, dv1 = 0.0;
    if (kk < nxm && field) {  // spectra: the field itself
      const double2 f = __ldg(reinterpret_cast<const double2 *>(field + col_off(g, j, i) + kk));
      dv0 = f.x;
      dv1 = (kk + 1 < nxm) ? f.y : 0.0;
    } else if (kk < nxm) {
      const int jp = wrap_inc(j, N);
      const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cip = col_off(g, j, ip);
      const double2 zi = __ldg(reinterpret_cast<const double2 *>(vz + cip + kk));
      const double2 zc = __ldg(reinterpret_cast<const double2 *>(vz + c + kk));
      const double2 yj = __ldg(reinterpret_cast<const double2 *>(vy + cjp + kk));
      const double2 yc = __ldg(reinterpret_cast<const double2 *>(vy + c + kk));
      const double2 xc = __ldg(reinterpret_cast<const double2 *>(vx + c + kk));
      dv0 = ((zi.x - zc.x) * g.dz + (yj.x - yc.x) * g.dy + (xc.y - xc.x) * ux.x) * usdtal;
      if (kk + 1 < nxm) {
        const double x2 = __ldg(vx + c + kk + 2);
        dv1 = ((zi.y - zc.y) * g.dz + (yj.y - yc.y) * g.dy + (x2 - xc.y) * ux.y) * usdtal;
      }
    }
    C z;
    z.x = (TS)dv0;
    z.y = (TS)dv1;
    T[tsw(j, q)] = z;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
  C x[N1];
#pragma unroll
  for (int m = 0; m < N1; ++m) x[m] = T[tsw(lane + 32 * m, p)];
  if constexpr (LT)
    warp_fft_lt<false, TS, N1>(x, lane, tw, stw);
  else
    warp_fft<false, TS, N1>(x, lane, tw);
  __syncthreads();
  const int rl = bitrev5(lane);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) T[tsw(k1 + N1 * rl, p)] = x[k1];
  __syncthreads();
  const TS norm = (TS)(1.0 / (nz_norm(g) * (double)g.nym));
  const TS half = (TS)0.5;
  for (int e = threadIdx.x; e < g.nyh * 16; e += blockDim.x) {
    const int ex = e & 15, ky = e >> 4;
    const int kk = k0 + ex;
    if (kk >= g.nxm) continue;
    const int q = ex >> 1;
    const C zk = T[tsw(ky, q)];
    const C zn = T[tsw(ky == 0 ? 0 : N - ky, q)];
    C X;
    if ((ex & 1) == 0) {
      X.x = (zk.x + zn.x) * half;
      X.y = (zk.y - zn.y) * half;
    } else {
      X.x = (zk.y + zn.y) * half;
      X.y = (zn.x - zk.x) * half;
    }
    X.x *= norm;
    X.y *= norm;
    spec[(size_t)(ky + (size_t)g.nyh * i) * g.ldxc + kk] = X;
  }
}

// 3-D and 4-D tiled tensor copies (no multicast): global -> shared completing on an mbarrier,
// and shared -> global in the issuing thread's bulk group.  `map` is a __grid_constant__ kernel
// parameter; the innermost coordinate must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *src) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
               : "memory");
}

// K2w, tensor-copy persistent form (FP64, single domain): the same divergence and y r2c transform
// of 16 x points at one z index (a tile), with the velocity rows staged by tiled TMA loads in
// chunks of 32 rows (vx with the 17th x point, vy with the row after the chunk, vz at i and at
// i + 1) instead of per-thread global loads, whose latency bounds k_div_fft_y_w.  Each block walks
// tiles blockIdx.x, + gridDim.x, ... as one stream of chunks with two or three in flight
// (div_nbuf), so the next tile's first chunks load while the current tile is transformed and
// stored.  The divergence's
// expression order, the packed tile, the transform and the output are those of k_div_fft_y_w, so
// the same bits.  The staging wait is bounded (bit 2 of *err, copies drained before the block
// exits).
struct DivMaps {
  CUtensorMap vx, vx2, vy, vyr, vz;  // 16 x 32 swizzled boxes; vx's 17th point; vy's next row
};
constexpr int kDivChunk = 32;                           // rows a chunk
constexpr uint32_t kDivChunkTx = 4 * 4096 + 512 + 128;  // bytes a chunk brings
constexpr int kDivChunkBytes = 17408;                   // a chunk buffer, 1024-aligned

// Blocks per SM that k_div_fft_y_wt's register cap allows, its dynamic shared memory with nb
// chunk buffers (alignment slack, chunks, the [N][8] tile, barriers, the lane-twiddle table
// where it keeps the blocks per SM), and the number of chunk buffers: a third where it costs no
// block per SM (N = 384, two blocks by registers), so that more of the next tile is in flight
// while a tile is transformed.
template <int N1>
__host__ __device__ constexpr int div_blocks_by_regs() {
  return (N1 <= 8) ? 3 : (N1 <= 16) ? 2 : 1;
}
template <int N1>
__host__ __device__ constexpr size_t div_smem(int nb) {
  const size_t core = 1024 + (size_t)nb * kDivChunkBytes + (size_t)32 * N1 * 128 + 32;  // 32: up to 4 barriers
  return core + (lane_table_fits(core, lane_table_bytes<N1>()) ? lane_table_bytes<N1>() : 0);
}
__host__ __device__ constexpr size_t div_min(size_t a, size_t b) { return a < b ? a : b; }
template <int N1>
__host__ __device__ constexpr int div_nbuf() {
  const size_t r = (size_t)div_blocks_by_regs<N1>(), b3 = div_smem<N1>(3), b2 = div_smem<N1>(2);
  return (b3 <= 227 * 1024 && div_min(r, (228 * 1024) / (b3 + 1024)) >= div_min(r, (228 * 1024) / (b2 + 1024))) ? 3
                                                                                                               : 2;
}

template <int N1>
__global__ void __launch_bounds__(256, div_blocks_by_regs<N1>())
    k_div_fft_y_wt(Geom g, Tables t, const StepCoef *__restrict__ sc_all, int ns, const __grid_constant__ DivMaps mp,
                   double2 *__restrict__ spec, const double2 *__restrict__ tw, int *__restrict__ err) {
  constexpr int N = 32 * N1;
  if (!inst_active(g, 0)) return;  // a single domain stopped by its step control
  extern __shared__ __align__(1024) unsigned char smem_k2t[];
  unsigned char *base = smem_k2t + ((1024u - (smem_u32(smem_k2t) & 1023u)) & 1023u);
  constexpr int NB = div_nbuf<N1>();  // chunk buffers
  double2 *T = reinterpret_cast<double2 *>(base + NB * kDivChunkBytes);  // [N][8] swizzled (tsw)
  uint64_t *bar = reinterpret_cast<uint64_t *>(T + N * 8);
  constexpr size_t kCore = 1024 + (size_t)NB * kDivChunkBytes + (size_t)N * 128 + 32;  // as div_smem
  constexpr bool LT = lane_table_fits(kCore, lane_table_bytes<N1>());
  double2 *stw = reinterpret_cast<double2 *>(base + kCore - 1024);  // lane twiddles (when LT)
  if constexpr (LT) fill_lane_twiddles<double, N1>(stw, tw);
  const int ntx = (g.nxm + 15) / 16;
  const int ntiles = ntx * g.nzm;
  const int mytiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nchunks = mytiles * N1;  // this block's chunk stream
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bar[b], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int sq) {  // thread 0: chunk sq of the stream into buffer sq % NB
    const int tile = blockIdx.x + (sq / N1) * gridDim.x, c = sq % N1, b = sq % NB;
    const int k0 = (tile % ntx) * 16, i = tile / ntx, ip = zinc(g, i);
    unsigned char *cb = base + b * kDivChunkBytes;
    const int j0 = kDivChunk * c;
    mbar_arrive_expect_tx(&bar[b], kDivChunkTx);
    tma_load_3d(cb, &mp.vx, k0, j0, i, &bar[b]);
    tma_load_3d(cb + 4096, &mp.vy, k0, j0, i, &bar[b]);
    tma_load_3d(cb + 8192, &mp.vz, k0, j0, i, &bar[b]);
    tma_load_3d(cb + 12288, &mp.vz, k0, j0, ip, &bar[b]);
    tma_load_3d(cb + 16384, &mp.vx2, k0 + 16, j0, i, &bar[b]);
    tma_load_3d(cb + 16896, &mp.vyr, k0, (j0 + kDivChunk) % N, i, &bar[b]);
  };
  if (tid == 0)
    for (int sq = 0; sq < NB && sq < nchunks; ++sq) issue(sq);
  const StepCoef sc = sc_all[sc_slot(g, 0, ns)];
  const double usdtal = 1.0 / (sc.dt * sc.al);
  const double norm = 1.0 / (nz_norm(g) * (double)g.nym);
  const int nxm = g.nxm;
  // thread (jl, q): row jl of each chunk, x points (kk, kk + 1) = (k0 + 2q, k0 + 2q + 1)
  const int q = tid & 7, jl = tid >> 3;
  const int lane = tid & 31, p = tid >> 5;
  for (int lt = 0; lt < mytiles; ++lt) {
    const int tile = blockIdx.x + lt * gridDim.x;
    const int k0 = (tile % ntx) * 16, i = tile / ntx;
    const int kk = k0 + 2 * q;
    const double2 ux = (kk < nxm) ? __ldg(reinterpret_cast<const double2 *>(t.udx3m + kk)) : make_double2(0.0, 0.0);
    for (int c = 0; c < N1; ++c) {
      const int sq = lt * N1 + c, b = sq % NB;
      const uint32_t par = (uint32_t)(sq / NB) & 1u;
      bool ok = mbar_wait(&bar[b], par, kSpinLimit);
      // test hook: the opposite phase is never completed here, so this wait always runs out
      if (g.wait_test_polls > 0) ok = ok && mbar_wait(&bar[b], par ^ 1u, g.wait_test_polls);
      if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicOr(err, 2);
        // copies in flight (this chunk and the next NB - 1) land before the block exits
        for (int d = 0; d < NB && sq + d < nchunks; ++d)
          mbar_wait(&bar[(sq + d) % NB], (uint32_t)((sq + d) / NB) & 1u, kDrainLimit);
        return;
      }
      const unsigned char *cb = base + b * kDivChunkBytes;
      // 16-byte chunk ch of row r of a swizzled 16 x 32 box at byte offset off
      auto at = [&](int off, int r, int ch) {
        return *reinterpret_cast<const double2 *>(cb + off + r * 128 + ((ch ^ (r & 7)) << 4));
      };
      double dv0 = 0.0, dv1 = 0.0;
      if (kk < nxm) {
        const double2 zi = at(12288, jl, q), zc = at(8192, jl, q);
        const double2 yj =
            (jl + 1 < kDivChunk) ? at(4096, jl + 1, q) : reinterpret_cast<const double2 *>(cb + 16896)[q];
        const double2 yc = at(4096, jl, q);
        const double2 xc = at(0, jl, q);
        dv0 = ((zi.x - zc.x) * g.dz + (yj.x - yc.x) * g.dy + (xc.y - xc.x) * ux.x) * usdtal;
        if (kk + 1 < nxm) {
          const double x2 = (q < 7) ? at(0, jl, q + 1).x : reinterpret_cast<const double2 *>(cb + 16384)[jl].x;
          dv1 = ((zi.y - zc.y) * g.dz + (yj.y - yc.y) * g.dy + (x2 - xc.y) * ux.y) * usdtal;
        }
      }
      T[tsw(kDivChunk * c + jl, q)] = make_double2(dv0, dv1);
      __syncthreads();  // chunk buffer b is free again
      if (tid == 0 && sq + NB < nchunks) issue(sq + NB);
    }
    double2 x[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) x[m] = T[tsw(lane + 32 * m, p)];
    if constexpr (LT)
      warp_fft_lt<false, double, N1>(x, lane, tw, stw);
    else
      warp_fft<false, double, N1>(x, lane, tw);
    __syncthreads();
    const int rl = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) T[tsw(k1 + N1 * rl, p)] = x[k1];
    __syncthreads();
    for (int e = tid; e < g.nyh * 16; e += blockDim.x) {
      const int ex = e & 15, ky = e >> 4;
      const int kx = k0 + ex;
      if (kx >= nxm) continue;
      const int qq = ex >> 1;
      const double2 zk = T[tsw(ky, qq)];
      const double2 zn = T[tsw(ky == 0 ? 0 : N - ky, qq)];
      double2 X;
      if ((ex & 1) == 0) {
        X.x = (zk.x + zn.x) * 0.5;
        X.y = (zk.y - zn.y) * 0.5;
      } else {
        X.x = (zk.y + zn.y) * 0.5;
        X.y = (zn.x - zk.x) * 0.5;
      }
      X.x *= norm;
      X.y *= norm;
      spec[(size_t)(ky + (size_t)g.nyh * i) * g.ldxc + kx] = X;
    }
    __syncthreads();  // the tile is read out before the next tile's divergence overwrites it
  }
}

// K3w / K5w: z c2c in place.  Block: 8 x points (8 warps) at one ky.
template <int N1, bool INV, typename TS>
__global__ void __launch_bounds__(256)
    k_fft_z_w(Geom g, typename Cplx<TS>::type *__restrict__ spec,
              const typename Cplx<TS>::type *__restrict__ tw) {
  using C = typename Cplx<TS>::type;
  constexpr int N = 32 * N1;
  extern __shared__ __align__(16) unsigned char smem_k3w[];
  C *s = reinterpret_cast<C *>(smem_k3w);  // [N][8], swizzled columns
  constexpr bool LT = lane_table_fits((size_t)N * 8 * sizeof(C), lane_table_bytes<N1, C>());
  C *stw = s + N * 8;  // lane twiddles (when LT)
  if constexpr (LT) fill_lane_twiddles<TS, N1>(stw, tw);
  const int k0 = blockIdx.x * 8, ky = blockIdx.y;
  const size_t zstride = (size_t)g.nyh * g.ldxc;
  C *base = spec + (size_t)ky * g.ldxc + k0;
  const int nvalid = min(8, g.nxm - k0);
  // the whole tile in flight at once: N1 asynchronous element copies per thread (256 threads,
  // N * 8 = 256 * N1 elements), zero-filled past nxm
#pragma unroll
  for (int it = 0; it < N1; ++it) {
    const int e = threadIdx.x + 256 * it;
    const int ex = e & 7, iz = e >> 3;
    const bool ok = ex < nvalid;
    cp_async_zfill<(int)sizeof(C)>(&s[iz * 8 + (ex ^ zsw(iz))], ok ? (const void *)(base + (size_t)iz * zstride + ex)
                                                                  : (const void *)base,
                                   ok);
  }
  cp_async_wait_all();
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  C x[N1];
#pragma unroll
  for (int m = 0; m < N1; ++m) {
    const int r = lane + 32 * m;
    x[m] = s[r * 8 + (w ^ zsw(r))];
  }
  if constexpr (LT)
    warp_fft_lt<INV, TS, N1>(x, lane, tw, stw);
  else
    warp_fft<INV, TS, N1>(x, lane, tw);
  __syncthreads();
  const int rl = bitrev5(lane);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    const int r = k1 + N1 * rl;
    s[r * 8 + (w ^ zsw(r))] = x[k1];
  }
  __syncthreads();
#pragma unroll 4
  for (int e = threadIdx.x; e < N * 8; e += blockDim.x) {
    const int ex = e & 7, iz = e >> 3;
    if (ex < nvalid) base[(size_t)iz * zstride + ex] = s[iz * 8 + (ex ^ zsw(iz))];
  }
}

// K3w / K5w, persistent form: each block transforms tiles t = blockIdx.x, + gridDim.x, ... (8 x
// points at one ky each, as k_fft_z_w) with two tile buffers: the next tile's asynchronous copies
// are in flight while the current tile is transformed and stored.  Same arithmetic as k_fft_z_w.
template <int N1, bool INV, typename TS>
__global__ void __launch_bounds__(256)
    k_fft_z_wp(Geom g, typename Cplx<TS>::type *__restrict__ spec,
               const typename Cplx<TS>::type *__restrict__ tw) {
  using C = typename Cplx<TS>::type;
  constexpr int N = 32 * N1;
  extern __shared__ __align__(16) unsigned char smem_k3p[];
  C *sb = reinterpret_cast<C *>(smem_k3p);  // [2][N][8], swizzled columns
  constexpr bool LT = lane_table_fits((size_t)2 * N * 8 * sizeof(C), lane_table_bytes<N1, C>());
  C *stw = sb + 2 * N * 8;  // lane twiddles (when LT)
  if constexpr (LT) fill_lane_twiddles<TS, N1>(stw, tw);
  const size_t zstride = (size_t)g.nyh * g.ldxc;
  const int ntx = (g.nxm + 7) / 8;
  const int ntiles = ntx * g.nyh;
  auto issue = [&](int tile, int b) {
    const int k0 = (tile % ntx) * 8, ky = tile / ntx;
    const C *base = spec + (size_t)ky * g.ldxc + k0;
    const int nvalid = min(8, g.nxm - k0);
    C *s = sb + (size_t)b * N * 8;
#pragma unroll
    for (int it = 0; it < N1; ++it) {
      const int e = threadIdx.x + 256 * it;
      const int ex = e & 7, iz = e >> 3;
      const bool ok = ex < nvalid;
      cp_async_zfill<(int)sizeof(C)>(&s[iz * 8 + (ex ^ zsw(iz))],
                                     ok ? (const void *)(base + (size_t)iz * zstride + ex) : (const void *)base, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile, 0);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int nt = tile + gridDim.x;
    if (nt < ntiles) {
      issue(nt, (it + 1) & 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    C *s = sb + (size_t)(it & 1) * N * 8;
    C x[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) {
      const int r = lane + 32 * m;
      x[m] = s[r * 8 + (w ^ zsw(r))];
    }
    if constexpr (LT)
      warp_fft_lt<INV, TS, N1>(x, lane, tw, stw);
    else
      warp_fft<INV, TS, N1>(x, lane, tw);
    __syncthreads();
    const int rl = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int r = k1 + N1 * rl;
      s[r * 8 + (w ^ zsw(r))] = x[k1];
    }
    __syncthreads();
    const int k0 = (tile % ntx) * 8, ky = tile / ntx;
    C *base = spec + (size_t)ky * g.ldxc + k0;
    const int nvalid = min(8, g.nxm - k0);
#pragma unroll 4
    for (int e = threadIdx.x; e < N * 8; e += blockDim.x) {
      const int ex = e & 7, iz = e >> 3;
      if (ex < nvalid) base[(size_t)iz * zstride + ex] = s[iz * 8 + (ex ^ zsw(iz))];
    }
    __syncthreads();  // this buffer is refilled by the copies issued in the next iteration but one
  }
}

// Shared-memory row of z index r = k1 + N1 * rl in k_fft_z_wt's output tile, where lane
// bitrev5(rl) of a warp holds it in register k1 after the warp FFT: row q + 8 a for
// r = a + 4 N1 q (q = rl >> 2, a = k1 + N1 (rl & 3)), the order in which the store tensor map
// (dimensions x, q, a) lays the tile out.  The row's low three bits are q, which differ between
// the eight lanes of a quarter warp, so with the 128-byte swizzle (16-byte chunk c of row R at
// c ^ (R & 7)) the write-back of one register across the warp is free of bank conflicts.
template <int N1>
__device__ __forceinline__ int zslot(int k1, int rl) {
  return ((rl >> 2) & 7) + 8 * (k1 + N1 * (rl & 3));
}

// K3w / K5w, tensor-copy persistent form: a tile (128 bytes of x at one ky, i.e. 8 x points of an
// FP64 spectrum or 16 of an FP32 one, whose warps then transform two adjacent columns each; all
// nzm z rows) comes in by one tiled TMA load and goes back by one tiled TMA store, so the load/store
// pipe carries only the transform's own shared-memory traffic (the per-thread asynchronous copies
// of k_fft_z_wp spend about a third of it, and one 1-D bulk copy per 128-byte row is bound by the
// copy engine's operation rate instead).  The load map views z as (z mod 32, z / 32) and fills the
// tile in z order; the store map views z as (z / 4 N1, z mod 4 N1) and reads the tile in zslot
// order, into which each warp writes its column's results in place (its own swizzled chunks, so no
// other warp is touched).  Both use the 128-byte swizzle; x points past nxm load as zeros and are
// not stored.  Two tiles in flight as in k_fft_z_wp; the same arithmetic, so the same bits.  The
// staging wait is bounded: a block that gives up sets bit 2 of *err, lets its copies land and
// exits.
template <int N1, bool INV, typename TS>
__global__ void __launch_bounds__(256)
    k_fft_z_wt(Geom g, const __grid_constant__ CUtensorMap ld_map, const __grid_constant__ CUtensorMap st_map,
               const typename Cplx<TS>::type *__restrict__ tw, int *__restrict__ err) {
  using C = typename Cplx<TS>::type;
  constexpr int N = 32 * N1;
  // a tile row is 128 bytes: 8 x points of double2, or 16 of float2 (two columns a warp)
  constexpr int CPW = 16 / (int)sizeof(C), XT = 8 * CPW;
  extern __shared__ __align__(1024) unsigned char smem_k3t[];
  // the 128-byte swizzle repeats every 1024 bytes: tiles start on such a boundary
  unsigned char *base = smem_k3t + ((1024u - (smem_u32(smem_k3t) & 1023u)) & 1023u);
  uint4 *sb = reinterpret_cast<uint4 *>(base);  // [2][N][8] 16-byte chunks
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + 2 * N * 8);
  constexpr bool LT = lane_table_fits(2 * N * 128 + 16 + 1024, lane_table_bytes<N1, C>());
  C *stw = reinterpret_cast<C *>(bar + 2);  // lane twiddles (when LT)
  if constexpr (LT) fill_lane_twiddles<TS, N1>(stw, tw);
  const int ntx = (g.nxm + XT - 1) / XT;
  const int ntiles = ntx * g.nyh;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int tile, int b) {  // thread 0
    const int k0 = (tile % ntx) * XT, ky = tile / ntx;
    mbar_arrive_expect_tx(&bar[b], 128u * N);
    tma_load_4d(sb + (size_t)b * N * 8, &ld_map, 2 * k0, 0, 0, ky, &bar[b]);
  };
  auto fft = [&](C(&x)[N1]) {
    if constexpr (LT)
      warp_fft_lt<INV, TS, N1>(x, lane, tw, stw);
    else
      warp_fft<INV, TS, N1>(x, lane, tw);
  };
  int tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile, 0);
  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int b = it & 1, nt = tile + gridDim.x;
    if (nt < ntiles) {
      // buffer b ^ 1 last held tile it - 1: its store must have read it before it is refilled
      if (tid == 0) bulk_wait_read();
      __syncthreads();
      if (tid == 0) issue(nt, b ^ 1);
    }
    const uint32_t par = (uint32_t)(it >> 1) & 1u;
    bool ok = mbar_wait(&bar[b], par, kSpinLimit);
    // test hook: the opposite phase is never completed here, so this wait always runs out
    if (g.wait_test_polls > 0) ok = ok && mbar_wait(&bar[b], par ^ 1u, g.wait_test_polls);
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicOr(err, 2);
      mbar_wait(&bar[b], par, kDrainLimit);  // copies in flight land before the block exits
      if (nt < ntiles) mbar_wait(&bar[b ^ 1], (uint32_t)((it + 1) >> 1) & 1u, kDrainLimit);
      break;
    }
    uint4 *s = sb + (size_t)b * N * 8;
    // chunk w of each row: the warp's column (FP64) or its two adjacent columns (FP32)
    C x[CPW][N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) {
      const int r = lane + 32 * m;
      if constexpr (CPW == 1) {
        x[0][m] = reinterpret_cast<const C *>(s)[r * 8 + (w ^ (r & 7))];
      } else {
        const float4 v = reinterpret_cast<const float4 *>(s)[r * 8 + (w ^ (r & 7))];
        x[0][m] = make_float2(v.x, v.y);
        x[CPW - 1][m] = make_float2(v.z, v.w);
      }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < CPW; ++c) fft(x[c]);
    const int rl = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int r = zslot<N1>(k1, rl);
      if constexpr (CPW == 1)
        reinterpret_cast<C *>(s)[r * 8 + (w ^ (r & 7))] = x[0][k1];
      else
        reinterpret_cast<float4 *>(s)[r * 8 + (w ^ (r & 7))] =
            make_float4(x[0][k1].x, x[0][k1].y, x[CPW - 1][k1].x, x[CPW - 1][k1].y);
    }
    fence_proxy_async_shared();
    __syncthreads();
    if (tid == 0) {
      tma_store_4d(&st_map, 2 * ((tile % ntx) * XT), 0, 0, tile / ntx, s);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_all();
}

// The two tensor maps of k_fft_z_wt over a spectrum [nzm][nyh][ldxc] of complex TS, viewed as
// TS: x (2 nxm, a 128-byte box row: 16 doubles or 32 floats), two z dimensions, ky.  Encoded through
// the driver's entry point (no driver library linked); false if that is unavailable or refuses.
using TmapEncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static TmapEncodeFn tmap_encoder() {
  static TmapEncodeFn fn = []() -> TmapEncodeFn {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<TmapEncodeFn>(f);
  }();
  return fn;
}

template <typename TS>
static bool fftz_tmaps(const Geom &g, int N1, typename Cplx<TS>::type *spec, CUtensorMap *ld, CUtensorMap *st) {
  using C = typename Cplx<TS>::type;
  TmapEncodeFn enc = tmap_encoder();
  if (!enc) return false;
  const CUtensorMapDataType dt = sizeof(TS) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint32_t bx = 128 / sizeof(TS);  // a 128-byte box row
  const cuuint64_t zb = (cuuint64_t)g.nyh * g.ldxc * sizeof(C);  // bytes between z rows
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const cuuint64_t ldim[4] = {(cuuint64_t)2 * g.nxm, 32, (cuuint64_t)N1, (cuuint64_t)g.nyh};
  const cuuint64_t lstr[3] = {zb, 32 * zb, (cuuint64_t)g.ldxc * sizeof(C)};
  const cuuint32_t lbox[4] = {bx, 32, (cuuint32_t)N1, 1};
  const cuuint64_t sdim[4] = {(cuuint64_t)2 * g.nxm, 8, (cuuint64_t)4 * N1, (cuuint64_t)g.nyh};
  const cuuint64_t sstr[3] = {(cuuint64_t)4 * N1 * zb, zb, (cuuint64_t)g.ldxc * sizeof(C)};
  const cuuint32_t sbox[4] = {bx, 8, (cuuint32_t)(4 * N1), 1};
  return enc(ld, dt, 4, spec, ldim, lstr, lbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
         enc(st, dt, 4, spec, sdim, sstr, sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// K6w: backward y c2r.  Block: 16 x points = 8 pairs (8 warps) at one z index i.  The half
// spectrum rows 0 .. N/2 of the 16 x points are staged with asynchronous copies (all in flight
// at once); each warp then builds its packed sequence straight from them.
template <int N1, typename TS>
__global__ void __launch_bounds__(256)
    k_ifft_y_w(Geom g, const typename Cplx<TS>::type *__restrict__ spec, TS *__restrict__ phi,
               const typename Cplx<TS>::type *__restrict__ tw) {
  using C = typename Cplx<TS>::type;
  constexpr int N = 32 * N1;
  constexpr int NH = N / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_k6w[];
  C *T = reinterpret_cast<C *>(smem_k6w);  // [N][8] swizzled (output transposition)
  C *R = T;                                 // [NH][16], element (jj, c) at jj*16 + (c ^ 2(jj & 7))
  const TS *Tr = reinterpret_cast<const TS *>(smem_k6w);
  constexpr bool LT = lane_table_fits((size_t)(N * 8 + 16) * sizeof(C), lane_table_bytes<N1, C>());
  C *stw = T + N * 8 + 16;  // lane twiddles (when LT)
  const int k0 = blockIdx.x * 16, i = blockIdx.y;
  if (!inst_active(g, i)) return;
  if constexpr (LT) fill_lane_twiddles<TS, N1>(stw, tw);
  const C *src0 = spec + (size_t)g.nyh * i * g.ldxc + k0;
  const int nvalid = min(16, g.nxm - k0);
  constexpr int kIt = (NH * 16 + 255) / 256;
#pragma unroll
  for (int it = 0; it < kIt; ++it) {
    const int e = threadIdx.x + 256 * it;
    if (e < NH * 16) {
      const int c = e & 15, jj = e >> 4;
      const bool ok = c < nvalid;
      cp_async_zfill<(int)sizeof(C)>(&R[jj * 16 + (c ^ ((jj & 7) << 1))],
                                     ok ? (const void *)(src0 + (size_t)jj * g.ldxc + c) : (const void *)src0, ok);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
  C x[N1];
#pragma unroll
  for (int m = 0; m < N1; ++m) {
    // row j of the full spectrum from row jj of the half spectrum (conjugate above N/2); the
    // pair (x points k0 + 2p, k0 + 2p + 1) packed as X + iY
    const int j = lane + 32 * m;
    const bool cj = (2 * j > N);
    const int jj = cj ? N - j : j;
    const int sw = (jj & 7) << 1;
    C X = R[jj * 16 + ((2 * p) ^ sw)], Y = R[jj * 16 + ((2 * p + 1) ^ sw)];
    if (cj) { X.y = -X.y; Y.y = -Y.y; }
    if (jj == 0 || 2 * jj == N) { X.y = 0; Y.y = 0; }
    x[m].x = X.x - Y.y;
    x[m].y = X.y + Y.x;
  }
  if constexpr (LT)
    warp_fft_lt<true, TS, N1>(x, lane, tw, stw);
  else
    warp_fft<true, TS, N1>(x, lane, tw);
  __syncthreads();
  const int rl = bitrev5(lane);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) T[tsw(k1 + N1 * rl, p)] = x[k1];
  __syncthreads();
  // the packed pair (re, im) of column p is phi at (k0 + 2p, k0 + 2p + 1): one vector store
  using V = typename Vec2<TS>::type;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * 8; e += blockDim.x) {
    const int q = e & 7, j = e >> 3;
    const int k = k0 + 2 * q;
    if (k < g.nxm) {
      const C v = T[tsw(j, q)];
      TS *dst = phi + col_off(g, j, i) + k;
      if (k + 1 < g.nxm)
        *reinterpret_cast<V *>(dst) = make_v2(v.x, v.y);
      else
        dst[0] = v.x;
    }
  }
  (void)Tr;
}

// K6w, tensor-copy persistent form (FP64 spectrum and phi, single domain, N <= 384): a tile
// (16 x points at one z index) is the half spectrum rows 0 .. N/2, brought in by two tiled TMA
// loads (8 x points each, 128-byte swizzle), and phi at its 16 x points of all N rows, sent out by
// one tiled TMA store whose map views y as (j / 4 N1, j mod 4 N1): the warps write the output
// tile over the staged input in zslot order, free of bank conflicts as in k_fft_z_wt.  The
// load/store pipe then carries only the transform's own shared-memory traffic.  Each block walks
// tiles blockIdx.x, + gridDim.x, ... with two tiles in flight.  The same arithmetic as
// k_ifft_y_w, so the same bits; x points past nxm load as zeros and are not stored.  The staging
// wait is bounded (bit 2 of *err, copies drained before the block exits).
template <int N1>
__global__ void __launch_bounds__(256)
    k_ifft_y_wt(Geom g, const __grid_constant__ CUtensorMap ld_map, const __grid_constant__ CUtensorMap st_map,
                const double2 *__restrict__ tw, int *__restrict__ err) {
  constexpr int N = 32 * N1;
  constexpr int NH = N / 2 + 1;
  constexpr int HB = (NH * 128 + 1023) / 1024 * 1024;  // bytes of one staged half, 1024-aligned
  static_assert(N * 128 <= 2 * HB, "the output tile fits over the staged halves");
  if (!inst_active(g, 0)) return;  // a single domain stopped by its step control
  extern __shared__ __align__(1024) unsigned char smem_k6t[];
  unsigned char *base = smem_k6t + ((1024u - (smem_u32(smem_k6t) & 1023u)) & 1023u);  // [2][2][HB]
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + 4 * HB);
  constexpr bool LT = lane_table_fits(4 * HB + 16 + 1024, lane_table_bytes<N1>());
  double2 *stw = reinterpret_cast<double2 *>(bar + 2);  // lane twiddles (when LT)
  if constexpr (LT) fill_lane_twiddles<double, N1>(stw, tw);
  const int ntx = (g.nxm + 15) / 16;
  const int ntiles = ntx * g.nzm;
  const int tid = threadIdx.x, lane = tid & 31, p = tid >> 5;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int tile, int b) {  // thread 0
    const int k0 = (tile % ntx) * 16, i = tile / ntx;
    const bool two = k0 + 8 < g.nxm;  // the second 8 x points hold data
    unsigned char *dst = base + (size_t)b * 2 * HB;
    mbar_arrive_expect_tx(&bar[b], (two ? 2u : 1u) * 128u * NH);
    tma_load_3d(dst, &ld_map, 2 * k0, 0, i, &bar[b]);
    if (two) tma_load_3d(dst + HB, &ld_map, 2 * k0 + 16, 0, i, &bar[b]);
  };
  int tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile, 0);
  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int b = it & 1, nt = tile + gridDim.x;
    if (nt < ntiles) {
      // buffer b ^ 1 last held tile it - 1: its store must have read it before it is refilled
      if (tid == 0) bulk_wait_read();
      __syncthreads();
      if (tid == 0) issue(nt, b ^ 1);
    }
    const uint32_t par = (uint32_t)(it >> 1) & 1u;
    bool ok = mbar_wait(&bar[b], par, kSpinLimit);
    // test hook: the opposite phase is never completed here, so this wait always runs out
    if (g.wait_test_polls > 0) ok = ok && mbar_wait(&bar[b], par ^ 1u, g.wait_test_polls);
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicOr(err, 2);
      mbar_wait(&bar[b], par, kDrainLimit);  // copies in flight land before the block exits
      if (nt < ntiles) mbar_wait(&bar[b ^ 1], (uint32_t)((it + 1) >> 1) & 1u, kDrainLimit);
      break;
    }
    unsigned char *tb = base + (size_t)b * 2 * HB;
    const double2 *Hp = reinterpret_cast<const double2 *>(tb + (p >> 2) * HB);  // the half of x point k0 + 2p
    const int c0 = (2 * p) & 7;  // its chunk within that half
    double2 x[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) {
      // row j of the full spectrum from row jj of the half spectrum (conjugate above N/2); the
      // pair (x points k0 + 2p, k0 + 2p + 1) packed as X + iY
      const int j = lane + 32 * m;
      const bool cj = (2 * j > N);
      const int jj = cj ? N - j : j;
      const int sw = jj & 7;
      double2 X = Hp[jj * 8 + (c0 ^ sw)], Y = Hp[jj * 8 + ((c0 + 1) ^ sw)];
      if (cj) {
        X.y = -X.y;
        Y.y = -Y.y;
      }
      if (jj == 0 || 2 * jj == N) {
        X.y = 0;
        Y.y = 0;
      }
      x[m].x = X.x - Y.y;
      x[m].y = X.y + Y.x;
    }
    if constexpr (LT)
      warp_fft_lt<true, double, N1>(x, lane, tw, stw);
    else
      warp_fft<true, double, N1>(x, lane, tw);
    __syncthreads();  // every warp has read its input before the tile is overwritten
    double2 *T = reinterpret_cast<double2 *>(tb);  // [N][8] output tile
    const int rl = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int r = zslot<N1>(k1, rl);
      T[r * 8 + (p ^ (r & 7))] = x[k1];  // chunk p of row r: phi at x points k0 + 2p, k0 + 2p + 1
    }
    fence_proxy_async_shared();
    __syncthreads();
    if (tid == 0) {
      tma_store_4d(&st_map, (tile % ntx) * 16, 0, 0, tile / ntx, T);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_all();
}

// The tensor maps of k_ifft_y_wt: the half spectrum [nzm][nyh][ldxc] of double2 viewed as
// doubles (x 2 nxm, ky, z; box 16 x nyh) and phi [nzm][nym][ldx] (x nxm, two y dimensions, z).
static bool ify_tmaps(const Geom &g, int N1, double2 *spec, double *phi, CUtensorMap *ld, CUtensorMap *st) {
  TmapEncodeFn enc = tmap_encoder();
  if (!enc || g.nyh > 256) return false;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const cuuint64_t ldim[3] = {(cuuint64_t)2 * g.nxm, (cuuint64_t)g.nyh, (cuuint64_t)g.nzm};
  const cuuint64_t lstr[2] = {(cuuint64_t)g.ldxc * sizeof(double2), (cuuint64_t)g.nyh * g.ldxc * sizeof(double2)};
  const cuuint32_t lbox[3] = {16, (cuuint32_t)g.nyh, 1};
  const cuuint64_t yb = (cuuint64_t)g.ldx * sizeof(double);  // bytes between y rows of phi
  const cuuint64_t sdim[4] = {(cuuint64_t)g.nxm, 8, (cuuint64_t)4 * N1, (cuuint64_t)g.nzm};
  const cuuint64_t sstr[3] = {(cuuint64_t)4 * N1 * yb, yb, (cuuint64_t)g.nym * yb};
  const cuuint32_t sbox[4] = {16, 8, (cuuint32_t)(4 * N1), 1};
  return enc(ld, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, spec, ldim, lstr, lbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
         enc(st, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, phi, sdim, sstr, sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ==========================================================================================
// Host-side launchers
// ==========================================================================================
static int pick_M(int nxm) {
  const int need = (nxm + 31) / 32;
  const int opts[] = {1, 2, 4, 8, 12, 16, 24, 32};
  for (int m : opts)
    if (m >= need) return m;
  return -1;
}

int cn_choose_M(int nxm) { return pick_M(nxm); }
size_t k1_smem_bytes(int ldx, int M, bool mixed, bool two_d) {
  (void)mixed;  // the RK3 histories are not staged
  return k1_smem(ldx, M, two_d);
}
size_t cn_tab_doubles(int M, int nsst) { return cn_table_size(M) * 3 * (size_t)nsst; }

cudaError_t launch_cn_tables(const LaunchCtx &L, const CnInputs &in) {
  CnBuildArgs a;
  for (int m = 0; m < 3; ++m) {
    a.mat[m].am = in.am[m];
    a.mat[m].ac = in.ac[m];
    a.mat[m].ap = in.ap[m];
    a.mat[m].off = in.off[m];
    a.mat[m].n = in.n[m];
    a.mat[m].temperature = (in.nmat == 3) ? (m == 2) : 1;
  }
  a.nmat = in.nmat;
  for (int s = 0; s < 3; ++s) {
    a.al[s] = in.al[s];
    a.ga[s] = in.ga[s];
    a.ro[s] = in.ro[s];
  }
  a.dt = in.dt;
  a.beta = in.beta;
  a.pect = in.pect;
  a.ren = in.ren;
  a.ns0 = in.ns0;
  a.nsub = in.nsub;
  a.dt_dev = in.dt_dev;
  a.inst = in.inst;
  a.active = in.active;
  const int nb = in.dt_dev ? in.ninst : 1;
  k_cn_tables<<<in.nmat * in.nsub * nb, 32, 0, L.stream>>>(a, in.M, in.tab, in.sc);
  return cudaGetLastError();
}

cudaError_t launch_explicit_implicit(const LaunchCtx &L, const SubstepBuffers &b, int ns) {
  const int ncol = L.g.nym * L.g.nzm;
  return L.mixed ? launch_k1_mixed(L, b, ns, L.k1_var, ncol) : launch_k1_fp64(L, b, ns, L.k1_var, ncol);
}

// ------------------------------------------------------------------------------------------
// K4, persistent form (FP64): each warp solves modes sys, sys + gridDim.x*W, ... and brings the
// next mode's right-hand side into shared memory with asynchronous copies (cp.async) while it
// solves the current one (two buffers a warp).  The mode-independent rows (amphk, apphk, acphk in
// chunk layout) are staged once a block and shared by its warps; the diagonal of a mode is formed
// from acphk as the one-mode kernel forms it, and the pinned (0,0) row is applied on the fly.
// Same arithmetic, in the same order, as k_tridiag_pressure.
// ------------------------------------------------------------------------------------------
template <int M, int WPB, typename TS>
__global__ void __launch_bounds__(WPB * 32, (WPB == 4) ? 4 : 2)
    k_tridiag_pressure_p(Geom g, Tables t, typename Cplx<TS>::type *__restrict__ spec, int *__restrict__ err) {
  using C = typename Cplx<TS>::type;
  extern __shared__ double smem_k4p[];
  constexpr int LD = chunk_ld(M);
  constexpr int FL = LD * M;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = g.nxm;
  double *sa = smem_k4p, *sc_ = sa + FL, *sacp = sa + 2 * FL;  // shared by the block
  TS *buf = reinterpret_cast<TS *>(sa + 3 * FL) + (size_t)warp * 4 * FL;  // [2][dr, di] of this warp
  for (int r = threadIdx.x; r < 32 * M; r += WPB * 32) {
    const int s = (r % M) * LD + r / M;
    sa[s] = (r < n && r > 0) ? __ldg(t.amphk + r) : 0.0;
    sc_[s] = (r < n - 1) ? __ldg(t.apphk + r) : 0.0;
    sacp[s] = (r < n) ? __ldg(t.acphk + r) : 0.0;
  }
  __syncthreads();
  const int nsys = g.nyh * g.nzm;
  const int stride = gridDim.x * WPB;
  int sys = blockIdx.x * WPB + warp;
  // the right-hand side of mode `m` into buffer `b`: rows r = lane + 32 tt, zero past nxm
  auto fetch = [&](int m, int b) {
    const C *colp = spec + (size_t)m * g.ldxc;
    TS *dr = buf + b * 2 * FL, *di = dr + FL;
#pragma unroll
    for (int tt = 0; tt < M; ++tt) {
      const int r = lane + 32 * tt;
      const int s = (r % M) * LD + r / M;
      const bool ok = r < n;
      const TS *src = ok ? &colp[r].x : &colp[0].x;
      cp_async_zfill<(int)sizeof(TS)>(&dr[s], src, ok);
      cp_async_zfill<(int)sizeof(TS)>(&di[s], src + 1, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (sys < nsys) fetch(sys, 0);
  bool bad = false;
  for (int it = 0; sys < nsys; ++it, sys += stride) {
    const int nxt = sys + stride;
    if (nxt < nsys) {
      fetch(nxt, (it + 1) & 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncwarp();
    TS *sdr = buf + (it & 1) * 2 * FL, *sdi = sdr + FL;
    const int ky = sys % g.nyh, kz = sys / g.nyh;
    const bool active = inst_active(g, kz);
    if (active) {
      const bool pin = (ky == 0 && (kz == 0 || g.batch));
      const double akj = __ldg(t.ak2 + (g.batch ? (size_t)kz * g.nym : 0) + ky);
      const double aki = g.batch ? 0.0 : __ldg(t.ak1 + kz);
      const int s0 = lane * M;
      // row s0 + q of this lane's chunk: the pinned row is phi = 0 (a = 0, b = 1, rhs 0)
      auto pinrow = [&](int q) { return pin && (s0 + q == n - 1); };
      auto diag = [&](int q) -> double {
        const int r = s0 + q;
        return (r < n && !pinrow(q)) ? (sacp[q * LD + lane] - akj - aki) * (1.0 + 1.0e-15) : 1.0;
      };
      auto aa = [&](int q) { return pinrow(q) ? 0.0 : sa[q * LD + lane]; };
      auto rr = [&](const TS *d, int q) { return pinrow(q) ? 0.0 : (double)d[q * LD + lane]; };
      double cp[M], yr[M], yi[M], v[M], w[M];
      cp[0] = 0.0; yr[0] = 0.0; yi[0] = 0.0; v[0] = 0.0; w[0] = 0.0;
#pragma unroll
      for (int q = 1; q < M; ++q) {
        const double a = aa(q), c = sc_[q * LD + lane];
        const double den = (q > 1) ? diag(q) - a * cp[q - 1] : diag(q);
        bad |= (den == 0.0);
        const double inv = 1.0 / den;
        cp[q] = c * inv;
        const double dr = rr(sdr, q), di = rr(sdi, q);
        if (q > 1) {
          yr[q] = (dr - a * yr[q - 1]) * inv;
          yi[q] = (di - a * yi[q - 1]) * inv;
          v[q] = -a * v[q - 1] * inv;
        } else {
          yr[q] = dr * inv;
          yi[q] = di * inv;
          v[q] = -a * inv;
        }
        w[q] = (q == M - 1) ? -c * inv : 0.0;
      }
#pragma unroll
      for (int q = M - 2; q >= 1; --q) {
        yr[q] -= cp[q] * yr[q + 1];
        yi[q] -= cp[q] * yi[q + 1];
        v[q] -= cp[q] * v[q + 1];
        w[q] -= cp[q] * w[q + 1];
      }
      const double as_ = aa(0), cs_ = sc_[lane];
      double A, B, Cc, Dr, Di;
      if constexpr (M == 1) {
        A = as_;
        B = diag(0);
        Cc = cs_;
        Dr = rr(sdr, 0);
        Di = rr(sdi, 0);
      } else {
        double vl = __shfl_up_sync(0xffffffffu, v[M - 1], 1);
        double wl = __shfl_up_sync(0xffffffffu, w[M - 1], 1);
        double yl_r = __shfl_up_sync(0xffffffffu, yr[M - 1], 1);
        double yl_i = __shfl_up_sync(0xffffffffu, yi[M - 1], 1);
        if (lane == 0) { vl = 0.0; wl = 0.0; yl_r = 0.0; yl_i = 0.0; }
        A = as_ * vl;
        B = diag(0) + as_ * wl + cs_ * v[1];
        Cc = (lane == 31) ? 0.0 : cs_ * w[1];
        Dr = rr(sdr, 0) - as_ * yl_r - cs_ * yr[1];
        Di = rr(sdi, 0) - as_ * yl_i - cs_ * yi[1];
      }
      bad |= (B == 0.0);
      const double rB = 1.0 / B;
      double al_ = A * rB, ga_ = Cc * rB, er = Dr * rB, ei = Di * rB;
#pragma unroll
      for (int h = 1; h < 32; h <<= 1) {
        double am = __shfl_up_sync(0xffffffffu, al_, h), gm = __shfl_up_sync(0xffffffffu, ga_, h);
        double ap = __shfl_down_sync(0xffffffffu, al_, h), gp = __shfl_down_sync(0xffffffffu, ga_, h);
        double erm = __shfl_up_sync(0xffffffffu, er, h), eim = __shfl_up_sync(0xffffffffu, ei, h);
        double erp = __shfl_down_sync(0xffffffffu, er, h), eip = __shfl_down_sync(0xffffffffu, ei, h);
        if (lane < h) { am = 0.0; gm = 0.0; erm = 0.0; eim = 0.0; }
        if (lane + h >= 32) { ap = 0.0; gp = 0.0; erp = 0.0; eip = 0.0; }
        const double dd = 1.0 - al_ * gm - ga_ * ap;
        bad |= (dd == 0.0);
        const double nrm = 1.0 / dd;
        er = (er - al_ * erm - ga_ * erp) * nrm;
        ei = (ei - al_ * eim - ga_ * eip) * nrm;
        const double na = -al_ * am * nrm, ng = -ga_ * gp * nrm;
        al_ = na;
        ga_ = ng;
      }
      double xnr = __shfl_down_sync(0xffffffffu, er, 1), xni = __shfl_down_sync(0xffffffffu, ei, 1);
      if (lane == 31) { xnr = 0.0; xni = 0.0; }
      __syncwarp();  // every lane has read its rows before any is overwritten
      // the results overwrite the inputs in the buffer, rounded to the spectrum's type once
      sdr[lane] = (TS)er;
      sdi[lane] = (TS)ei;
#pragma unroll
      for (int q = 1; q < M; ++q) {
        sdr[q * LD + lane] = (TS)(yr[q] + v[q] * er + w[q] * xnr);
        sdi[q * LD + lane] = (TS)(yi[q] + v[q] * ei + w[q] * xni);
      }
      __syncwarp();
      C *colp = spec + (size_t)sys * g.ldxc;
#pragma unroll 1
      for (int tt = 0; tt < M; ++tt) {
        const int r = lane + 32 * tt;
        if (r < n) {
          const int s = (r % M) * LD + r / M;
          C o;
          o.x = sdr[s];
          o.y = sdi[s];
          colp[r] = o;
        }
      }
    }
    __syncwarp();  // this buffer is refilled two modes from now
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (bad) atomicOr(err, 1);
}

// Persistent grid: as many blocks as can be resident at once, no more than there are modes.
template <typename K>
static int k4p_grid(K kern, int nsys, int wpb, size_t smem) {
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, wpb * 32, smem) != cudaSuccess || per < 1) per = 1;
  return std::max(1, std::min((nsys + wpb - 1) / wpb, nsm * per));
}

template <int M, typename TS>
static cudaError_t launch_k4p_M(const LaunchCtx &L, void *spec, int *err) {
  constexpr int W = (M >= 16) ? 2 : 4;
  const int nsys = L.g.nyh * L.g.nzm;
  const size_t smem = (size_t)3 * chunk_ld(M) * M * sizeof(double) + (size_t)4 * W * chunk_ld(M) * M * sizeof(TS);
  auto kern = k_tridiag_pressure_p<M, W, TS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<k4p_grid(kern, nsys, W, smem), W * 32, smem, L.stream>>>(L.g, L.t, (typename Cplx<TS>::type *)spec, err);
  return cudaGetLastError();
}

template <int M, typename TS>
static cudaError_t launch_k4_M(const LaunchCtx &L, void *spec, int *err) {
  constexpr int W = (M >= 16) ? 2 : 4;
  const int nsys = L.g.nyh * L.g.nzm;
  const size_t smem = (size_t)W * (M <= 8 ? 5 : 4) * chunk_ld(M) * M * sizeof(double);
  auto kern = k_tridiag_pressure<M, W, TS>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(nsys + W - 1) / W, W * 32, smem, L.stream>>>(L.g, L.t, (typename Cplx<TS>::type *)spec, err);
  return cudaGetLastError();
}

template <typename TS>
static cudaError_t launch_k4_T(const LaunchCtx &L, void *spec, int *err) {
  if (L.k4_var == 1) {  // the persistent prefetching form (the autotuner's pick)
    switch (L.M) {
      case 1: return launch_k4p_M<1, TS>(L, spec, err);
      case 2: return launch_k4p_M<2, TS>(L, spec, err);
      case 4: return launch_k4p_M<4, TS>(L, spec, err);
      case 8: return launch_k4p_M<8, TS>(L, spec, err);
      case 12: return launch_k4p_M<12, TS>(L, spec, err);
      case 16: return launch_k4p_M<16, TS>(L, spec, err);
      case 24: return launch_k4p_M<24, TS>(L, spec, err);
      case 32: return launch_k4p_M<32, TS>(L, spec, err);
    }
    return cudaErrorInvalidValue;
  }
  switch (L.M) {
    case 1: return launch_k4_M<1, TS>(L, spec, err);
    case 2: return launch_k4_M<2, TS>(L, spec, err);
    case 4: return launch_k4_M<4, TS>(L, spec, err);
    case 8: return launch_k4_M<8, TS>(L, spec, err);
    case 12: return launch_k4_M<12, TS>(L, spec, err);
    case 16: return launch_k4_M<16, TS>(L, spec, err);
    case 24: return launch_k4_M<24, TS>(L, spec, err);
    case 32: return launch_k4_M<32, TS>(L, spec, err);
  }
  return cudaErrorInvalidValue;
}

// The tensor maps of k_div_fft_y_wt over the intermediate velocities [nzm][nym][ldx] (doubles):
// 16 x 32 swizzled boxes of vx (x extent nx, so its 17th point is the wall value at nxm), vy and
// vz (x extent nxm), two x points of vx past the tile, and one unswizzled row of vy.
static bool div_tmaps(const Geom &g, const double *vx, const double *vy, const double *vz, DivMaps *m) {
  TmapEncodeFn enc = tmap_encoder();
  if (!enc || g.nym < kDivChunk) return false;
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint64_t yb = (cuuint64_t)g.ldx * sizeof(double);
  const cuuint64_t str[2] = {yb, (cuuint64_t)g.nym * yb};
  const cuuint64_t dimx[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.nym, (cuuint64_t)g.nzm};
  const cuuint64_t dimm[3] = {(cuuint64_t)g.nxm, (cuuint64_t)g.nym, (cuuint64_t)g.nzm};
  const cuuint32_t box[3] = {16, (cuuint32_t)kDivChunk, 1}, box2[3] = {2, (cuuint32_t)kDivChunk, 1},
                   boxr[3] = {16, 1, 1};
  auto one = [&](CUtensorMap *t, const double *f, const cuuint64_t *dim, const cuuint32_t *bx, bool swz) {
    return enc(t, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(f), dim, str, bx, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swz ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  return one(&m->vx, vx, dimx, box, true) && one(&m->vx2, vx, dimx, box2, false) && one(&m->vy, vy, dimm, box, true) &&
         one(&m->vyr, vy, dimm, boxr, false) && one(&m->vz, vz, dimm, box, true);
}

// Launch helpers for the warp-FFT kernels: 8 warps per block, a [N][8] complex tile each
// (y transforms: 16 x points as 8 pairs; z transforms: 8 x points).
template <typename TS, int N1>
static cudaError_t launch_w_n1(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st) {
  using C = typename Cplx<TS>::type;
  const Geom &g = L.g;
  C *spec = (C *)b.spec;
  constexpr int N = 32 * N1;
  if (st == Stage::DivFftY || st == Stage::IfftY) {
    const size_t sm = (size_t)N * 8 * sizeof(C);
    dim3 grid((g.nxm + 15) / 16, g.nzm);
    // tensor copies (FP64 single domain); a field's transform (spectra) takes the per-thread form
    if (st == Stage::DivFftY && L.div_var == 1 && !b.fft_field) {
      if constexpr (!std::is_same<TS, double>::value) {
        return cudaErrorInvalidValue;
      } else {
        if (g.batch) return cudaErrorInvalidValue;
        const size_t sm2 = div_smem<N1>(div_nbuf<N1>());
        if (sm2 > (size_t)227 * 1024) return cudaErrorInvalidValue;
        DivMaps mp;
        if (!div_tmaps(g, b.vx_o, b.vy_o, b.vz_o, &mp)) return cudaErrorInvalidValue;
        auto kern = k_div_fft_y_wt<N1>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 148, per = 1;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm2) != cudaSuccess || per < 1) per = 1;
        const int ntiles = ((g.nxm + 15) / 16) * g.nzm;
        kern<<<std::max(1, std::min(ntiles, nsm * per)), 256, sm2, L.stream>>>(g, L.t, b.sc, ns, mp, spec,
                                                                              (const double2 *)L.twy, b.err);
      }
    } else if (st == Stage::DivFftY) {
      const size_t smt = sm + (lane_table_fits(sm, lane_table_bytes<N1, C>()) ? lane_table_bytes<N1, C>() : 0);
      auto kern = k_div_fft_y_w<N1, TS>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt);
      kern<<<grid, 256, smt, L.stream>>>(g, L.t, b.sc, ns, b.vx_o, b.vy_o, b.vz_o, spec, (const C *)L.twy,
                                         b.fft_field);
    } else if (L.ify_var == 1) {  // tensor copies (FP64 single domain, N <= 384)
      if constexpr (!std::is_same<TS, double>::value || N1 > 12) {
        return cudaErrorInvalidValue;
      } else {
        if (g.batch) return cudaErrorInvalidValue;
        constexpr int NH = N / 2 + 1;
        const size_t hb = (size_t)(NH * 128 + 1023) / 1024 * 1024;
        size_t sm6 = 4 * hb + 2 * sizeof(uint64_t) + 1024;  // two tiles of two halves
        if (lane_table_fits(sm6, lane_table_bytes<N1>())) sm6 += lane_table_bytes<N1>();
        CUtensorMap ld_map, st_map;
        if (!ify_tmaps(g, N1, spec, (double *)b.phi, &ld_map, &st_map)) return cudaErrorInvalidValue;
        auto kern = k_ifft_y_wt<N1>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm6);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 148, per = 1;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm6) != cudaSuccess || per < 1) per = 1;
        const int ntiles = ((g.nxm + 15) / 16) * g.nzm;
        kern<<<std::max(1, std::min(ntiles, nsm * per)), 256, sm6, L.stream>>>(g, ld_map, st_map,
                                                                              (const double2 *)L.twy, b.err);
      }
    } else {
      // the staged half spectrum [N/2 + 1][16] is 16 elements larger than the [N][8] tile
      size_t sm6 = (size_t)(N * 8 + 16) * sizeof(C);
      if (lane_table_fits(sm6, lane_table_bytes<N1, C>())) sm6 += lane_table_bytes<N1, C>();
      auto kern = k_ifft_y_w<N1, TS>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm6);
      kern<<<grid, 256, sm6, L.stream>>>(g, spec, (TS *)b.phi, (const C *)L.twy);
    }
    return cudaGetLastError();
  }
  const size_t sm = (size_t)N * 8 * sizeof(C);
  if (L.fftz_var == 2) {  // persistent, tiles moved by tensor copies
    // two 1024-byte aligned tiles of N x 128 bytes, the barriers, the alignment slack
    size_t smb = (size_t)2 * N * 128 + 2 * sizeof(uint64_t) + 1024;
    if (lane_table_fits(smb, lane_table_bytes<N1, C>())) smb += lane_table_bytes<N1, C>();
    if (smb > (size_t)227 * 1024 || 4 * N1 > 256) return cudaErrorInvalidValue;  // two tiles do not fit
    CUtensorMap ld_map, st_map;
    if (!fftz_tmaps<TS>(g, N1, spec, &ld_map, &st_map)) return cudaErrorInvalidValue;
    auto kern = (st == Stage::FftZFwd) ? k_fft_z_wt<N1, false, TS> : k_fft_z_wt<N1, true, TS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, smb) != cudaSuccess || per < 1) per = 1;
    constexpr int XT = 128 / (int)sizeof(C);  // x points a tile
    const int ntiles = ((g.nxm + XT - 1) / XT) * g.nyh;
    kern<<<std::max(1, std::min(ntiles, nsm * per)), 256, smb, L.stream>>>(g, ld_map, st_map, (const C *)L.twz,
                                                                          b.err);
    return cudaGetLastError();
  }
  if (L.fftz_var == 1) {  // persistent, double-buffered tiles
    if (2 * sm > (size_t)227 * 1024) return cudaErrorInvalidValue;  // two tiles do not fit
    const size_t smp = 2 * sm + (lane_table_fits(2 * sm, lane_table_bytes<N1, C>()) ? lane_table_bytes<N1, C>() : 0);
    auto kern = (st == Stage::FftZFwd) ? k_fft_z_wp<N1, false, TS> : k_fft_z_wp<N1, true, TS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, smp) != cudaSuccess || per < 1) per = 1;
    const int ntiles = ((g.nxm + 7) / 8) * g.nyh;
    kern<<<std::max(1, std::min(ntiles, nsm * per)), 256, smp, L.stream>>>(g, spec, (const C *)L.twz);
    return cudaGetLastError();
  }
  dim3 grid((g.nxm + 7) / 8, g.nyh);
  const size_t smt = sm + (lane_table_fits(sm, lane_table_bytes<N1, C>()) ? lane_table_bytes<N1, C>() : 0);
  auto kern = (st == Stage::FftZFwd) ? k_fft_z_w<N1, false, TS> : k_fft_z_w<N1, true, TS>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt);
  kern<<<grid, 256, smt, L.stream>>>(g, spec, (const C *)L.twz);
  return cudaGetLastError();
}

// The warp FFT handles N = 32*{1,2,3,4,6,8,12,16,24,32}; returns false otherwise.
template <typename TS>
static bool launch_warp_fft(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st, cudaError_t *err) {
  const int N = (st == Stage::FftZFwd || st == Stage::FftZInv) ? L.g.nzm : L.g.nym;
  if (N % 32 != 0) return false;
  switch (N / 32) {
    case 1: *err = launch_w_n1<TS, 1>(L, b, ns, st); return true;
    case 2: *err = launch_w_n1<TS, 2>(L, b, ns, st); return true;
    case 3: *err = launch_w_n1<TS, 3>(L, b, ns, st); return true;
    case 4: *err = launch_w_n1<TS, 4>(L, b, ns, st); return true;
    case 6: *err = launch_w_n1<TS, 6>(L, b, ns, st); return true;
    case 8: *err = launch_w_n1<TS, 8>(L, b, ns, st); return true;
    case 12: *err = launch_w_n1<TS, 12>(L, b, ns, st); return true;
    case 16: *err = launch_w_n1<TS, 16>(L, b, ns, st); return true;
    case 24: *err = launch_w_n1<TS, 24>(L, b, ns, st); return true;
    case 32: *err = launch_w_n1<TS, 32>(L, b, ns, st); return true;
  }
  return false;
}

template <typename TS>
static cudaError_t launch_stage_T(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st) {
  using C = typename Cplx<TS>::type;
  const Geom &g = L.g;
  C *spec = (C *)b.spec;
  const C *twy = (const C *)L.twy;
  const C *twz = (const C *)L.twz;
  if (L.warp_fft && (st == Stage::DivFftY || st == Stage::IfftY ||
                     ((st == Stage::FftZFwd || st == Stage::FftZInv) && g.nzm > 1 && !g.batch))) {
    cudaError_t e = cudaSuccess;
    if (launch_warp_fft<TS>(L, b, ns, st, &e)) return e;
  }
  switch (st) {
    case Stage::DivFftY: {  // K2 divergence + forward y FFT
      const int TX = L.tx_y;
      const size_t smem = (size_t)TX * g.nym * sizeof(C);  // 2 buffers of TX/2 sequences
      dim3 grid((g.nxm + TX - 1) / TX, g.nzm);
      if (TX == 8) {
        cudaFuncSetAttribute(k_div_fft_y<8, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_div_fft_y<8, TS><<<grid, 256, smem, L.stream>>>(g, L.t, b.sc, ns, b.vx_o, b.vy_o, b.vz_o, spec,
                                                          L.plan_y, twy, b.fft_field);
      } else if (TX == 4) {
        cudaFuncSetAttribute(k_div_fft_y<4, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_div_fft_y<4, TS><<<grid, 256, smem, L.stream>>>(g, L.t, b.sc, ns, b.vx_o, b.vy_o, b.vz_o, spec,
                                                          L.plan_y, twy, b.fft_field);
      } else {
        cudaFuncSetAttribute(k_div_fft_y<2, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_div_fft_y<2, TS><<<grid, 256, smem, L.stream>>>(g, L.t, b.sc, ns, b.vx_o, b.vy_o, b.vz_o, spec,
                                                          L.plan_y, twy, b.fft_field);
      }
      return cudaGetLastError();
    }
    case Stage::FftZFwd:
    case Stage::FftZInv: {  // K3 / K5 z FFT (none for one 2-D domain or a batch of them)
      if (g.nzm == 1 || g.batch) return cudaSuccess;
      const int TXZ = L.tx_z;
      const size_t smem = (size_t)2 * TXZ * g.nzm * sizeof(C);
      dim3 grid((g.nxm + TXZ - 1) / TXZ, g.nyh);
      const bool inv = (st == Stage::FftZInv);
#define AFID_FFTZ(TXv, INVv)                                                                       \
  do {                                                                                             \
    cudaFuncSetAttribute(k_fft_z<TXv, INVv, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    k_fft_z<TXv, INVv, TS><<<grid, 256, smem, L.stream>>>(g, spec, L.plan_z, twz);                 \
  } while (0)
      if (TXZ == 8) { if (inv) AFID_FFTZ(8, true); else AFID_FFTZ(8, false); }
      else if (TXZ == 4) { if (inv) AFID_FFTZ(4, true); else AFID_FFTZ(4, false); }
      else { if (inv) AFID_FFTZ(2, true); else AFID_FFTZ(2, false); }
#undef AFID_FFTZ
      return cudaGetLastError();
    }
    case Stage::Tridiag:  // K4
      return launch_k4_T<TS>(L, b.spec, b.err);
    case Stage::IfftY: {  // K6 backward y FFT -> phi
      const int TX = L.tx_y;
      const size_t smem = (size_t)TX * g.nym * sizeof(C);
      dim3 grid((g.nxm + TX - 1) / TX, g.nzm);
      TS *phi = (TS *)b.phi;
      if (TX == 8) {
        cudaFuncSetAttribute(k_ifft_y<8, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_ifft_y<8, TS><<<grid, 256, smem, L.stream>>>(g, spec, phi, L.plan_y, twy);
      } else if (TX == 4) {
        cudaFuncSetAttribute(k_ifft_y<4, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_ifft_y<4, TS><<<grid, 256, smem, L.stream>>>(g, spec, phi, L.plan_y, twy);
      } else {
        cudaFuncSetAttribute(k_ifft_y<2, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_ifft_y<2, TS><<<grid, 256, smem, L.stream>>>(g, spec, phi, L.plan_y, twy);
      }
      return cudaGetLastError();
    }
    case Stage::Correct: {  // K7 projection + pressure update, two x points a thread
      const int pairs = (g.nxm + 1) / 2;
      const int bx = (pairs >= 128) ? 128 : ((pairs + 31) / 32) * 32;
      const int by = 256 / bx;
      dim3 block(bx, by);
      dim3 grid((pairs + bx - 1) / bx, (g.nym + by - 1) / by, g.nzm);
      k_correct<TS><<<grid, block, 0, L.stream>>>(g, L.t, b.sc, ns, b.vx_o, b.vy_o, b.vz_o, b.vx, b.vy,
                                                  b.vz, b.pr, (const TS *)b.phi);
      return cudaGetLastError();
    }
    case Stage::ExplicitImplicit:
      return launch_explicit_implicit(L, b, ns);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st) {
  if (st == Stage::ExplicitImplicit) return launch_explicit_implicit(L, b, ns);
  return L.mixed ? launch_stage_T<float>(L, b, ns, st) : launch_stage_T<double>(L, b, ns, st);
}

// dst[r*dld + k] = src[r*sld + k], k < width: between the padded device layout and a packed
// staging copy (host transfers then run as one linear copy per field).
__global__ void k_repack(const double *__restrict__ src, int sld, double *__restrict__ dst, int dld, int width,
                         size_t rows) {
  const size_t n = rows * (size_t)width;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / width;
    const int k = (int)(e - r * width);
    dst[r * dld + k] = src[r * sld + k];
  }
}

cudaError_t launch_repack(cudaStream_t st, const double *src, int sld, double *dst, int dld, int width,
                          size_t rows) {
  const size_t n = rows * (size_t)width;
  const int nb = (int)std::min<size_t>((n + 255) / 256, (size_t)148 * 16);
  k_repack<<<nb, 256, 0, st>>>(src, sld, dst, dld, width, rows);
  return cudaGetLastError();
}

static int reduce_blocks(const Geom &g) {
  const long long ncol = (long long)g.nym * g.nzm;
  long long nb = (ncol + 7) / 8;  // 8 warps per block, one column per warp per pass
  if (nb > 148 * 8) nb = 148 * 8;
  if (nb < 1) nb = 1;
  return (int)nb;
}

cudaError_t launch_max_reduce(const LaunchCtx &L, bool div, const double *vx, const double *vy,
                              const double *vz, unsigned long long *out) {
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), L.stream);
  const int nb = reduce_blocks(L.g);
  if (div)
    k_max_reduce<true><<<nb, 256, 0, L.stream>>>(L.g, L.t, vx, vy, vz, out);
  else
    k_max_reduce<false><<<nb, 256, 0, L.stream>>>(L.g, L.t, vx, vy, vz, out);
  return cudaGetLastError();
}

cudaError_t launch_globals(const LaunchCtx &L, const double *vx, const double *vy, const double *vz,
                           const double *temp, double *partial, double *out3) {
  const int nb = reduce_blocks(L.g);
  k_globals_partial<<<nb, 256, 0, L.stream>>>(L.g, L.t, vx, vy, vz, temp, partial);
  k_sum_partials<<<1, 256, 0, L.stream>>>(partial, nb, out3);
  return cudaGetLastError();
}

int globals_partial_blocks(const Geom &g) { return reduce_blocks(g); }

}  // namespace afid
