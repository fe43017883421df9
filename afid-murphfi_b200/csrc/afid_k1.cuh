// afid_k1.cuh — K1: ExplicitTerms{VX,VY,VZ,Temp} + ImplicitAndUpdate* + SolveImpEqnUpdate_*
// fused per x-column (template; instantiated for FP64 in afid_k1_fp64.cu and for FP32 explicit
// terms in afid_k1_mixed.cu).  Thread shapes per M (threads per column x rows per thread) are
// listed in kK1Shapes; the autotuner picks one per context.
#pragma once
#include <algorithm>

#include "afid_device.cuh"
#include "afid_internal.h"

namespace afid {

// Loads by cache policy.  H = 0: read-only data through the non-coherent path (__ldg) and the
// RK3 histories by plain loads.  H = 1: the tables every block reads (metric coefficients, CN
// factors) are kept in L1 with the evict_last priority, and the data each block reads once (RK3
// histories, single-row neighbours) bypasses L1 (no_allocate), so the streaming data does not
// evict the tables.  H = 2 (tld only): the tables sit in shared memory; plain loads.
template <int H> __device__ __forceinline__ double tld(const double *p) {
  if constexpr (H == 2) {  // tables staged in shared memory (k_explicit_implicit_p)
    return *p;
  } else if constexpr (H != 0) {
    double v;
    asm("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}
template <int H> __device__ __forceinline__ double nld(const double *p) {
  if constexpr (H != 0) {
    double v;
    asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
  } else {
    return __ldg(p);
  }
}
// Read-write streaming data (the histories, rewritten later by the same thread): coherent loads.
template <int H> __device__ __forceinline__ double sld(const double *p) {
  if constexpr (H != 0) {
    double v;
    asm volatile("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
  } else {
    return *p;
  }
}
template <int H> __device__ __forceinline__ double sld(const float *p) {
  if constexpr (H != 0) {
    float v;
    asm volatile("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return (double)v;
  } else {
    return (double)*p;
  }
}

// Doubles per CN factor table (one matrix, one substep); layout in afid_kernels.cu.
__host__ __device__ inline size_t cn_table_size(int M) { return 192 * (size_t)M + 18 * 32; }

// The forward-elimination factors of one lane (a_q, 1/b'_q for q < M), loaded ahead of the
// solve by a caller that has a barrier to hide their latency behind (cn_solve_chunk with PRE).
template <int M, int H = 0>
struct CnFwd {
  double a[M], inv[M];
  __device__ __forceinline__ void load(const double *__restrict__ T, int lane) {
#pragma unroll
    for (int q = 1; q < M; ++q) {
      inv[q] = tld<H>(T + 64 * M + q * 32 + lane);
      if (q >= 2) a[q] = tld<H>(T + 32 * M + q * 32 + lane);
    }
  }
};

// Solve one column whose scaled RHS sits in s[q*32 + lane] (chunk layout); the solution
// overwrites it.  Constant-matrix version using the tables above.  PRE: the forward factors
// come from `fw` (loaded earlier) instead of from the table.
template <int M, int LD = 32, int H = 0, bool PRE = false>
__device__ __forceinline__ void cn_solve_chunk(double *__restrict__ s, const double *__restrict__ T,
                                               int lane, const CnFwd<M, H> *fw = nullptr) {
  const double *Ta = T + 32 * M, *Tinv = T + 64 * M, *Tcp = T + 96 * M, *Tv = T + 128 * M,
               *Tw = T + 160 * M, *Tl = T + 192 * M;
  double y[M];
#pragma unroll
  for (int q = 0; q < M; ++q) y[q] = s[q * LD + lane];
  if constexpr (M > 1) {
    y[1] = y[1] * (PRE ? fw->inv[1] : tld<H>(Tinv + 32 + lane));
#pragma unroll
    for (int q = 2; q < M; ++q)
      y[q] = (y[q] - (PRE ? fw->a[q] : tld<H>(Ta + q * 32 + lane)) * y[q - 1]) *
             (PRE ? fw->inv[q] : tld<H>(Tinv + q * 32 + lane));
#pragma unroll
    for (int q = M - 2; q >= 1; --q) y[q] = y[q] - tld<H>(Tcp + q * 32 + lane) * y[q + 1];
  }
  double D;
  if constexpr (M > 1) {
    double yprev = __shfl_up_sync(0xffffffffu, y[M - 1], 1);
    if (lane == 0) yprev = 0.0;
    D = y[0] - tld<H>(Tl + lane) * yprev - tld<H>(Tl + 32 + lane) * y[1];
  } else {
    D = y[0];
  }
  double delta = D * tld<H>(Tl + 64 + lane);
#pragma unroll
  for (int lev = 0, h = 1; lev < 5; ++lev, h <<= 1) {
    double dm = __shfl_up_sync(0xffffffffu, delta, h);
    double dp = __shfl_down_sync(0xffffffffu, delta, h);
    if (lane < h) dm = 0.0;
    if (lane + h >= 32) dp = 0.0;
    delta = (delta - tld<H>(Tl + 96 + lev * 32 + lane) * dm - tld<H>(Tl + 256 + lev * 32 + lane) * dp) *
            tld<H>(Tl + 416 + lev * 32 + lane);
  }
  double xnext = __shfl_down_sync(0xffffffffu, delta, 1);
  if (lane == 31) xnext = 0.0;
  s[lane] = delta;
#pragma unroll
  for (int q = 1; q < M; ++q)
    s[q * LD + lane] = y[q] + tld<H>(Tv + q * 32 + lane) * delta + tld<H>(Tw + q * 32 + lane) * xnext;
}

// Two columns with the same matrix (s0, s1: chunk layout as above) solved by one warp: every
// factor is loaded once and applied to both right-hand sides, in the same operation order as
// cn_solve_chunk (so each solution is bitwise the same as a single solve).
template <int M, int LD = 32, int H = 0>
__device__ __forceinline__ void cn_solve_chunk2(double *__restrict__ s0, double *__restrict__ s1,
                                                const double *__restrict__ T, int lane) {
  const double *Ta = T + 32 * M, *Tinv = T + 64 * M, *Tcp = T + 96 * M, *Tv = T + 128 * M,
               *Tw = T + 160 * M, *Tl = T + 192 * M;
  double y[M], z[M];
#pragma unroll
  for (int q = 0; q < M; ++q) {
    y[q] = s0[q * LD + lane];
    z[q] = s1[q * LD + lane];
  }
  if constexpr (M > 1) {
    const double i1 = tld<H>(Tinv + 32 + lane);
    y[1] = y[1] * i1;
    z[1] = z[1] * i1;
#pragma unroll
    for (int q = 2; q < M; ++q) {
      const double a = tld<H>(Ta + q * 32 + lane), iv = tld<H>(Tinv + q * 32 + lane);
      y[q] = (y[q] - a * y[q - 1]) * iv;
      z[q] = (z[q] - a * z[q - 1]) * iv;
    }
#pragma unroll
    for (int q = M - 2; q >= 1; --q) {
      const double cp = tld<H>(Tcp + q * 32 + lane);
      y[q] = y[q] - cp * y[q + 1];
      z[q] = z[q] - cp * z[q + 1];
    }
  }
  double Dy, Dz;
  if constexpr (M > 1) {
    double yprev = __shfl_up_sync(0xffffffffu, y[M - 1], 1);
    double zprev = __shfl_up_sync(0xffffffffu, z[M - 1], 1);
    if (lane == 0) yprev = zprev = 0.0;
    const double l0 = tld<H>(Tl + lane), l1 = tld<H>(Tl + 32 + lane);
    Dy = y[0] - l0 * yprev - l1 * y[1];
    Dz = z[0] - l0 * zprev - l1 * z[1];
  } else {
    Dy = y[0];
    Dz = z[0];
  }
  const double l2 = tld<H>(Tl + 64 + lane);
  double dy = Dy * l2, dz = Dz * l2;
#pragma unroll
  for (int lev = 0, h = 1; lev < 5; ++lev, h <<= 1) {
    double ym = __shfl_up_sync(0xffffffffu, dy, h), yp = __shfl_down_sync(0xffffffffu, dy, h);
    double zm = __shfl_up_sync(0xffffffffu, dz, h), zp = __shfl_down_sync(0xffffffffu, dz, h);
    if (lane < h) ym = zm = 0.0;
    if (lane + h >= 32) yp = zp = 0.0;
    const double lm = tld<H>(Tl + 96 + lev * 32 + lane), lp = tld<H>(Tl + 256 + lev * 32 + lane),
                 li = tld<H>(Tl + 416 + lev * 32 + lane);
    dy = (dy - lm * ym - lp * yp) * li;
    dz = (dz - lm * zm - lp * zp) * li;
  }
  double ynext = __shfl_down_sync(0xffffffffu, dy, 1), znext = __shfl_down_sync(0xffffffffu, dz, 1);
  if (lane == 31) ynext = znext = 0.0;
  s0[lane] = dy;
  s1[lane] = dz;
#pragma unroll
  for (int q = 1; q < M; ++q) {
    const double v = tld<H>(Tv + q * 32 + lane), w = tld<H>(Tw + q * 32 + lane);
    s0[q * LD + lane] = y[q] + v * dy + w * ynext;
    s1[q * LD + lane] = z[q] + v * dz + w * znext;
  }
}

// ------------------------------------------------------------------------------------------
// Explicit terms + RHS, one (k, j, i) point each.  Expressions follow the reference loop
// bodies term by term; TE is the arithmetic type of the explicit terms.  The operands are
// x-columns staged in shared memory: c = (j,i), jp/jm = (j+-1,i), ip/im = (j,i+-1),
// The diagonal neighbours (vy at (j+1,i-1), vz at (j-1,i+1)) and the pressure at (j-1,i) and
// (j,i-1) are read at row k only, so they arrive as values (zd, yd, pjm, pim), not columns.
// ------------------------------------------------------------------------------------------
struct ColV {
  const double *c, *jp, *jm, *ip, *im, *d;
};

template <typename TE> __device__ __forceinline__ TE cv(double v) { return (TE)v; }

// In 2-D (TWO_D: the z neighbours are the cell itself) every z-difference term is zero by
// construction; those terms are left out instead of being evaluated to zero.

// The per-row table operands of the four explicit terms (they depend on the row k only), loaded
// together from global or shared memory before the terms that use them.
struct RowTab {
  double idxm, idxc, udx3c, udx3m, ap3ck, ac3ck, am3ck, ap3sk, ac3sk, am3sk, ap3ssk, ac3ssk, am3ssk;
};
template <int H> __device__ __forceinline__ RowTab row_tab(const Tables &t, int k) {
  RowTab r;
  r.idxm = (k >= 1) ? tld<H>(t.idx + k - 1) : 0.0;  // read by the vx terms only, k >= 1
  r.idxc = tld<H>(t.idx + k);
  r.udx3c = tld<H>(t.udx3c + k);
  r.udx3m = tld<H>(t.udx3m + k);
  r.ap3ck = tld<H>(t.ap3ck + k);
  r.ac3ck = tld<H>(t.ac3ck + k);
  r.am3ck = tld<H>(t.am3ck + k);
  r.ap3sk = tld<H>(t.ap3sk + k);
  r.ac3sk = tld<H>(t.ac3sk + k);
  r.am3sk = tld<H>(t.am3sk + k);
  r.ap3ssk = tld<H>(t.ap3ssk + k);
  r.ac3ssk = tld<H>(t.ac3ssk + k);
  r.am3ssk = tld<H>(t.am3ssk + k);
  return r;
}

// ExplicitTermsVX.F90:30-127 + ImplicitAndUpdateVX.F90:39-66, k = 1..nxm-1 (0-based)
template <typename TE, bool TWO_D, bool SAL, int H = 0>
__device__ __forceinline__ double rhs_vx(const Geom &g, const RowTab &r, const StepCoef &sc, int k,
                                         const ColV &X, const ColV &Y, const ColV &Z, const ColV &T,
                                         const ColV &P, double ru, TE &qout, double sb) {
  const int km = k - 1, kp = k + 1;
  const TE udy = (TE)(g.dy * 0.25), udz = (TE)(g.dz * 0.25);
  const TE udyq = (TE)g.udyq_re, udzq = (TE)g.udzq_re;
  const TE idxm = cv<TE>(r.idxm), idxc = cv<TE>(r.idxc);
  const TE udx3c = cv<TE>(r.udx3c);
  const TE vxc = cv<TE>(X.c[k]);
  const TE vxkp = cv<TE>(X.c[kp]), vxkm = cv<TE>(X.c[km]);
  const TE vxip = cv<TE>(X.ip[k]), vxim = cv<TE>(X.im[k]);
  const TE vxjp = cv<TE>(X.jp[k]), vxjm = cv<TE>(X.jm[k]);
  TE hxz = (TE)0, dzzvx = (TE)0;
  if constexpr (!TWO_D) {
    hxz = udx3c * udz *
          ((idxm * cv<TE>(Z.ip[km]) + idxc * cv<TE>(Z.ip[k])) * (vxip + vxc) -
           (idxm * cv<TE>(Z.c[km]) + idxc * cv<TE>(Z.c[k])) * (vxc + vxim));
    dzzvx = (vxim - (TE)2.0 * vxc + vxip) * udzq;
  }
  const TE hxy = udx3c * udy *
                 ((idxm * cv<TE>(Y.jp[km]) + idxc * cv<TE>(Y.jp[k])) * (vxjp + vxc) -
                  (idxm * cv<TE>(Y.c[km]) + idxc * cv<TE>(Y.c[k])) * (vxc + vxjm));
  const TE hxx = ((vxkp + vxc) * (vxkp + vxc) - (vxc + vxkm) * (vxc + vxkm)) * udx3c * (TE)0.25;
  const TE dyyvx = (vxjm - (TE)2.0 * vxc + vxjp) * udyq;
  TE qcap = TWO_D ? (-(hxx + hxy) + dyyvx) : (-(hxx + hxy + hxz) + dyyvx + dzzvx);
  if (g.gaxis == 1) {
    const TE tempit = (TE)g.active_t * (TE)0.5 * (cv<TE>(T.c[k]) + cv<TE>(T.c[km]));
    qcap = qcap + (TE)g.byct * tempit;
    if constexpr (SAL) qcap = qcap - (TE)sb;  // AddSalBuoyancy(qcap)
  }
  const double alre = sc.alre;
  const double udx3 = sc.al * r.udx3c;
  const double dxxvx = X.c[kp] * r.ap3ck + X.c[k] * r.ac3ck + X.c[km] * r.am3ck;
  const double dxp = (P.c[k] - P.c[km]) * udx3;
  qout = qcap;
  return (sc.ga * (double)qcap + sc.ro * ru + alre * dxxvx - dxp) * sc.dt;
}

// ExplicitTermsVY.F90:23-122 + ImplicitAndUpdateVY.F90:28-80, k = 0..nxm-1
template <typename TE, bool TWO_D, bool SAL, int H = 0>
__device__ __forceinline__ double rhs_vy(const Geom &g, const RowTab &r, const StepCoef &sc, int k,
                                         const ColV &X, const ColV &Y, const ColV &Z, const ColV &T,
                                         const ColV &P, double zd, double pjm, double ru, TE &qout,
                                         double sb) {
  const int kmm = (k == 0) ? 0 : k - 1;
  const int kpp = (k == g.nxm - 1) ? k : k + 1;
  const int kp = k + 1;
  const TE udy = (TE)(g.dy * 0.25), udz = (TE)(g.dz * 0.25);
  const TE udyq = (TE)g.udyq_re, udzq = (TE)g.udzq_re;
  const TE c = cv<TE>(Y.c[k]);
  const TE vyjp = cv<TE>(Y.jp[k]), vyjm = cv<TE>(Y.jm[k]);
  const TE vyip = cv<TE>(Y.ip[k]), vyim = cv<TE>(Y.im[k]);
  const TE hyx = ((cv<TE>(X.c[kp]) + cv<TE>(X.jm[kp])) * (cv<TE>(Y.c[kpp]) + c) -
                  (cv<TE>(X.c[k]) + cv<TE>(X.jm[k])) * (c + cv<TE>(Y.c[kmm]))) *
                 cv<TE>(r.udx3m) * (TE)0.25;
  const TE hyy = ((vyjp + c) * (vyjp + c) - (vyjm + c) * (vyjm + c)) * udy;
  const TE dyyvy = (vyjp - (TE)2.0 * c + vyjm) * udyq;
  TE dph;
  if constexpr (TWO_D) {
    dph = -(hyx + hyy) + dyyvy + (TE)g.gy;
  } else {
    const TE hyz = ((vyip + c) * (cv<TE>(Z.ip[k]) + cv<TE>(zd)) - (c + vyim) * (cv<TE>(Z.c[k]) + cv<TE>(Z.jm[k]))) *
                   udz;
    const TE dzzvy = (vyip - (TE)2.0 * c + vyim) * udzq;
    dph = -(hyx + hyy + hyz) + dyyvy + dzzvy + (TE)g.gy;
  }
  if (g.gaxis == 2) {
    const TE tempit = (TE)g.active_t * (TE)0.5 * (cv<TE>(T.c[k]) + cv<TE>(T.jm[k]));
    dph = dph + (TE)g.byct * tempit;
    if constexpr (SAL) dph = dph - (TE)sb;  // AddSalBuoyancy(dph)
  }
  const double alre = sc.alre;
  const double udyp = g.dy * sc.al;
  const double amm = r.am3sk, acc = r.ac3sk, app = r.ap3sk;
  const double cd = Y.c[k];
  double dxxvy;
  if (k == 0)
    dxxvy = Y.c[kpp] * app + cd * acc - (acc + app) * g.xminusu * g.inslws;
  else if (k == g.nxm - 1)
    dxxvy = -(acc + amm) * g.xplusu * g.inslwn + cd * acc + Y.c[kmm] * amm;
  else
    dxxvy = Y.c[kpp] * app + cd * acc + Y.c[kmm] * amm;
  const double dyp = (P.c[k] - pjm) * udyp;
  qout = dph;
  return (sc.ga * (double)dph + sc.ro * ru + alre * dxxvy - dyp) * sc.dt;
}

// ExplicitTermsVZ.F90:23-118 + ImplicitAndUpdateVZ.F90:38-69, k = 0..nxm-1
template <typename TE, bool TWO_D, bool SAL, int H = 0>
__device__ __forceinline__ double rhs_vz(const Geom &g, const RowTab &r, const StepCoef &sc, int k,
                                         const ColV &X, const ColV &Y, const ColV &Z, const ColV &T,
                                         const ColV &P, double yd, double pim, double ru, TE &qout,
                                         double sb) {
  const int kmm = (k == 0) ? 0 : k - 1;
  const int kpp = (k == g.nxm - 1) ? k : k + 1;
  const int kp = k + 1;
  const TE udy = (TE)(g.dy * 0.25), udz = (TE)(g.dz * 0.25);
  const TE udyq = (TE)g.udyq_re, udzq = (TE)g.udzq_re;
  const TE c = cv<TE>(Z.c[k]);
  const TE vzip = cv<TE>(Z.ip[k]), vzim = cv<TE>(Z.im[k]);
  const TE vzjp = cv<TE>(Z.jp[k]), vzjm = cv<TE>(Z.jm[k]);
  const TE hzy = ((cv<TE>(Y.jp[k]) + cv<TE>(yd)) * (vzjp + c) - (cv<TE>(Y.c[k]) + cv<TE>(Y.im[k])) * (c + vzjm)) *
                 udy;
  const TE hzx = ((cv<TE>(X.c[kp]) + cv<TE>(X.im[kp])) * (cv<TE>(Z.c[kpp]) + c) -
                  (cv<TE>(X.c[k]) + cv<TE>(X.im[k])) * (c + cv<TE>(Z.c[kmm]))) *
                 cv<TE>(r.udx3m) * (TE)0.25;
  const TE dyyvz = (vzjp - (TE)2.0 * c + vzjm) * udyq;
  TE dq;
  if constexpr (TWO_D) {
    dq = -(hzx + hzy) + dyyvz;
  } else {
    const TE hzz = ((vzip + c) * (vzip + c) - (vzim + c) * (vzim + c)) * udz;
    const TE dzzvz = (vzip - (TE)2.0 * c + vzim) * udzq;
    dq = -(hzx + hzy + hzz) + dyyvz + dzzvz;
  }
  if (g.gaxis == 3) {
    const TE tempit = (TE)g.active_t * (TE)0.5 * (cv<TE>(T.c[k]) + cv<TE>(T.im[k]));
    dq = dq + (TE)g.byct * tempit;
    if constexpr (SAL) dq = dq - (TE)sb;  // AddSalBuoyancy(dq)
  }
  const double alre = sc.alre;
  const double amm = r.am3sk, acc = r.ac3sk, app = r.ap3sk;
  const double dxxvz = Z.c[kpp] * app + Z.c[k] * acc + Z.c[kmm] * amm;
  qout = dq;
  if constexpr (TWO_D) {
    return (sc.ga * (double)dq + sc.ro * ru + alre * dxxvz) * sc.dt;
  } else {
    const double dzp = (P.c[k] - pim) * g.dz * sc.al;
    return (sc.ga * (double)dq + sc.ro * ru + alre * dxxvz - dzp) * sc.dt;
  }
}

// ExplicitTermsTemp.F90:22-77 + ImplicitAndUpdateTemp.F90:33-66, k = 0..nxm-1
template <typename TE, bool TWO_D, int H = 0>
__device__ __forceinline__ double rhs_temp(const Geom &g, const RowTab &r, const StepCoef &sc, int k,
                                           const ColV &X, const ColV &Y, const ColV &Z, const ColV &T,
                                           double tbp, double ttp, double ru, TE &qout) {
  const TE udz = (TE)(g.dz * 0.5), udy = (TE)(g.dy * 0.5);
  const TE udzq = (TE)g.udzq_pe, udyq = (TE)g.udyq_pe;
  const TE tc = cv<TE>(T.c[k]);
  const TE ux = cv<TE>(r.udx3m);
  TE htx;
  if (k == 0)
    htx = (cv<TE>(X.c[1]) * (cv<TE>(T.c[1]) + tc) - cv<TE>(X.c[0]) * (TE)2.0 * (TE)tbp) * (TE)0.5 * ux;
  else if (k == g.nxm - 1)
    htx = (cv<TE>(X.c[k + 1]) * (TE)2.0 * (TE)ttp - cv<TE>(X.c[k]) * (tc + cv<TE>(T.c[k - 1]))) * (TE)0.5 * ux;
  else
    htx = (cv<TE>(X.c[k + 1]) * (cv<TE>(T.c[k + 1]) + tc) - cv<TE>(X.c[k]) * (tc + cv<TE>(T.c[k - 1]))) *
          (TE)0.5 * ux;
  const TE tip = cv<TE>(T.ip[k]), tim = cv<TE>(T.im[k]);
  const TE tjp = cv<TE>(T.jp[k]), tjm = cv<TE>(T.jm[k]);
  const TE hty = (cv<TE>(Y.jp[k]) * (tjp + tc) - cv<TE>(Y.c[k]) * (tc + tjm)) * udy;
  const TE dyyt = (tjp - (TE)2.0 * tc + tjm) * udyq;
  TE hro;
  if constexpr (TWO_D) {
    hro = -(htx + hty) + dyyt;
  } else {
    const TE htz = (cv<TE>(Z.ip[k]) * (tip + tc) - cv<TE>(Z.c[k]) * (tc + tim)) * udz;
    const TE dzzt = (tip - (TE)2.0 * tc + tim) * udzq;
    hro = -(htx + hty + htz) + dyyt + dzzt;
  }
  const double alpec = sc.alpec;
  const double tcd = T.c[k];
  double dxxt;
  if (k == 0)
    dxxt = T.c[1] * r.ap3ssk + tcd * r.ac3ssk - (r.ap3ssk + r.ac3ssk) * tbp * g.tfixs;
  else if (k == g.nxm - 1)
    dxxt = tcd * r.ac3ssk + T.c[k - 1] * r.am3ssk - (r.am3ssk + r.ac3ssk) * ttp * g.tfixn;
  else
    dxxt = T.c[k + 1] * r.ap3ssk + tcd * r.ac3ssk + T.c[k - 1] * r.am3ssk;
  qout = hro;
  return (sc.ga * (double)hro + sc.ro * ru + alpec * dxxt) * sc.dt;
}

// Number of x-columns K1 stages per (j,i) column (FP64 state): vx 5, vy 5, vz 5, temp 5, pr 1
// (the diagonal vy/vz neighbours and the pressure neighbours are read at one row each and go
// straight to registers).  In 2-D (nzm = 1, or a batch of 2-D instances) the z neighbours are the
// column itself, leaving vx, vy, vz, temp at (j, j+1, j-1) and pr at j: 13 columns.  The four
// centre columns come first; after the explicit phase the others are dead and hold the CN
// right-hand sides.
constexpr int kK1StateCols = 21;
constexpr int kK1StateCols2D = 13;
constexpr int kK1Centre = 4;

__host__ __device__ inline size_t k1_stage_bytes(int ldx, bool two_d) {
  return (size_t)(two_d ? kK1StateCols2D : kK1StateCols) * ldx * sizeof(double);
}
// Staged columns sit at a compile-time stride of 32 M + 8 doubles (>= ldx = round_up(nxm+1, 8)
// because nxm <= 32 M, and equal to it when nxm = 32 M), so every operand address is one base
// register plus an immediate offset.
__host__ __device__ constexpr int k1_col_stride(int M) { return 32 * M + 8; }
// Dynamic shared memory of K1: the staged columns, or the centre columns plus the four RHS
// arrays in chunk layout, whichever is larger.
__host__ __device__ inline size_t k1_smem(int ldx, int M, bool two_d) {
  (void)ldx;
  const int cs = k1_col_stride(M);
  const size_t rhs = (size_t)kK1Centre * cs * sizeof(double) + (size_t)4 * chunk_ld(M) * M * sizeof(double);
  const size_t st = (size_t)(two_d ? kK1StateCols2D : kK1StateCols) * cs * sizeof(double);
  return st > rhs ? st : rhs;
}

// K1: a block owns one (j,i) column.  One thread issues 1-D TMA bulk copies of the needed
// x-columns (contiguous runs of ldx doubles) into shared memory, completing on an mbarrier;
// then TPC threads each compute the four explicit terms and RHS of RPT cells from shared memory
// (the RK3 histories come straight from global memory and are updated in place), and, after a
// barrier, put the scaled RHS into the chunk layout (row r at (r%M)*LD + r/M) over the dead
// neighbour columns.  Four warps run the partitioned CN solves, and every thread adds the
// increments to the staged centre values and stores the intermediate fields.
// CAP: register cap for at least 16 (CAP = 1) or 32 (CAP = 2) resident warps per SM, i.e. <= 128
// or <= 64 registers a thread; with CAP = 0 the compiler may use more registers for fewer
// resident blocks.
template <int CAP, int TPC>
constexpr int k1_min_blocks() {
  return CAP == 0 ? 1 : ((CAP == 1 ? 512 : 1024) / TPC > 1 ? (CAP == 1 ? 512 : 1024) / TPC : 1);
}
template <int M, int TPC, int RPT, typename TE, bool TWO_D, int CAP, bool SAL, int POL>
__global__ void __launch_bounds__(TPC, k1_min_blocks<CAP, TPC>())
    k_explicit_implicit(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
                        const double *__restrict__ cn_tab, const double *__restrict__ vx,
                        const double *__restrict__ vy, const double *__restrict__ vz,
                        const double *__restrict__ temp, const double *__restrict__ pr,
                        TE *__restrict__ rux, TE *__restrict__ ruy, TE *__restrict__ ruz,
                        TE *__restrict__ rut, double *__restrict__ vx_o, double *__restrict__ vy_o,
                        double *__restrict__ vz_o, double *__restrict__ temp_o, int *__restrict__ err) {
  constexpr int LD = chunk_ld(M);
  constexpr int FLD = LD * M;
  constexpr int H = POL & 1;  // cache policy of the global loads (tld / nld / sld above)
  // rows of a thread: tc + TPC p (strided), or RPT tc + p (adjacent, POL bit 2), so that the
  // k - 1 / k + 1 operands of one row are the centre operands of the next
  constexpr bool ADJ = (POL & 4) != 0;
  extern __shared__ __align__(128) unsigned char smem_k1[];
  __shared__ uint64_t bar;
  Geom g = g0;
  const int ldx = g.ldx;
  double *cols = reinterpret_cast<double *>(smem_k1);
  constexpr int CS = k1_col_stride(M);
  double *s_rhs = cols + (size_t)kK1Centre * CS;  // over the neighbour columns, after they are used
  const int tc = threadIdx.x;
  const int colid = blockIdx.x;
  const int j = colid % g.nym, i = colid / g.nym;
  if (!inst_active(g, i)) {
    // An idle batch slot keeps its state: the temperature moves buffers every substep.
    const size_t c = col_off(g, j, i);
    for (int k = tc; k < g.nx; k += TPC) temp_o[c + k] = temp[c + k];
    return;
  }
  bind_instance(g, i);
  const int jp = wrap_inc(j, g.nym), jm = wrap_dec(j, g.nym);
  const int ip = zinc(g, i), im = zdec(g, i);
  const size_t c0 = col_off(g, j, i);
  if (tc == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tc == 0) {
    const size_t oc = c0, ojp = col_off(g, jp, i), ojm = col_off(g, jm, i), oip = col_off(g, j, ip),
                 oim = col_off(g, j, im), ojpim = col_off(g, jp, im), ojmip = col_off(g, jm, ip);
    const uint32_t cb = (uint32_t)ldx * sizeof(double);
    mbar_arrive_expect_tx(&bar, (uint32_t)k1_stage_bytes(ldx, TWO_D));
    (void)ojpim;
    (void)ojmip;
    if constexpr (TWO_D) {
      const double *src[kK1StateCols2D] = {vx + oc,   vy + oc,    vz + oc, temp + oc,  // 0-3 centre
                                           vx + ojp,  vx + ojm,                        // 4-5
                                           vy + ojp,  vy + ojm,                        // 6-7
                                           vz + ojp,  vz + ojm,                        // 8-9
                                           temp + ojp, temp + ojm,                     // 10-11
                                           pr + oc};                                   // 12
#pragma unroll
      for (int q = 0; q < kK1StateCols2D; ++q) bulk_g2s(cols + (size_t)q * CS, src[q], cb, &bar);
    } else {
      const double *src[kK1StateCols] = {vx + oc,    vy + oc,    vz + oc,    temp + oc,   // 0-3
                                         vx + ojp,   vx + ojm,   vx + oip,   vx + oim,    // 4-7
                                         vy + ojp,   vy + ojm,   vy + oip,   vy + oim,    // 8-11
                                         vz + ojp,   vz + ojm,   vz + oip,   vz + oim,    // 12-15
                                         temp + ojp, temp + ojm, temp + oip, temp + oim,  // 16-19
                                         pr + oc};                                        // 20
#pragma unroll
      for (int q = 0; q < kK1StateCols; ++q) bulk_g2s(cols + (size_t)q * CS, src[q], cb, &bar);
    }
  }
  // single-row operands: diagonal neighbours (3-D) and pressure neighbours, to registers
  const size_t o_jm = col_off(g, jm, i), o_im = col_off(g, j, im);
  const size_t o_jpim = col_off(g, jp, im), o_jmip = col_off(g, jm, ip);
  // the RK3 histories go straight to registers; their loads overlap the staging copies
  double uu[RPT][4], vv[RPT][4];  // RK3 histories; {vz(j-1,i+1), vy(j+1,i-1), pr(j-1), pr(i-1)}
  double sbv[SAL ? RPT : 1];       // salinity buoyancy bycs * salc of each row (SAL only)
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = ADJ ? RPT * tc + p : tc + TPC * p;
    const bool in = k < g.nxm;
    uu[p][0] = (in && k >= 1) ? sld<H>(rux + c0 + k) : 0.0;
    uu[p][1] = in ? sld<H>(ruy + c0 + k) : 0.0;
    uu[p][2] = in ? sld<H>(ruz + c0 + k) : 0.0;
    uu[p][3] = in ? sld<H>(rut + c0 + k) : 0.0;
    if constexpr (TWO_D) {
      vv[p][0] = 0.0;  // taken from the staged vz(j-1) / vy(j+1) columns below
      vv[p][1] = 0.0;
      vv[p][3] = 0.0;  // pr(i-1) is the centre column
    } else {
      vv[p][0] = in ? nld<H>(vz + o_jmip + k) : 0.0;
      vv[p][1] = in ? nld<H>(vy + o_jpim + k) : 0.0;
      vv[p][3] = in ? nld<H>(pr + o_im + k) : 0.0;
    }
    vv[p][2] = in ? nld<H>(pr + o_jm + k) : 0.0;
    if constexpr (SAL) sbv[p] = in ? g.bycs * nld<H>(g.salc + c0 + k) : 0.0;
  }
  const int slot = sc_slot(g, i, ns);
  const size_t tsz = cn_table_size(M);
  const double *TX = cn_tab + (size_t)(slot * 3 + 0) * tsz;
  const double *TY = cn_tab + (size_t)(slot * 3 + 1) * tsz;
  const double *TT = cn_tab + (size_t)(slot * 3 + 2) * tsz;
  // POL bit 3: the first row's table operands and CN row scalings are loaded before the wait as
  // well, so their latency overlaps the staging copies (all rows' would not fit the registers)
  constexpr bool EARLY = (POL & 8) != 0;
  RowTab rte;
  double rse[3];
  if constexpr (EARLY) {
    const int k = ADJ ? RPT * tc : tc;
    if (k < g.nxm) {
      rte = row_tab<H>(t, k);
      rse[0] = (k >= 1) ? tld<H>(TX + k - 1) : 0.0;
      rse[1] = tld<H>(TY + k);
      rse[2] = tld<H>(TT + k);
    }
  }

  bool ok = mbar_wait(&bar, 0, kSpinLimit);
  // test hook: phase 1 of the barrier is never completed, so this wait always runs out
  if (g.wait_test_polls > 0) ok = ok && mbar_wait(&bar, 1, g.wait_test_polls);
  if (!__syncthreads_and(ok)) {
    if (tc == 0) atomicOr(err, 2);
    mbar_wait(&bar, 0, kDrainLimit);  // let copies in flight land before the block exits
    return;
  }
  auto C = [&](int q) { return (const double *)(cols + q * CS); };
  // {centre, j+1, j-1, i+1, i-1, diagonal}; in 2-D the i+-1 columns are the centre's
  const ColV X = TWO_D ? ColV{C(0), C(4), C(5), C(0), C(0), nullptr} : ColV{C(0), C(4), C(5), C(6), C(7), nullptr};
  const ColV Y = TWO_D ? ColV{C(1), C(6), C(7), C(1), C(1), nullptr} : ColV{C(1), C(8), C(9), C(10), C(11), nullptr};
  const ColV Z = TWO_D ? ColV{C(2), C(8), C(9), C(2), C(2), nullptr} : ColV{C(2), C(12), C(13), C(14), C(15), nullptr};
  const ColV T = TWO_D ? ColV{C(3), C(10), C(11), C(3), C(3), nullptr} : ColV{C(3), C(16), C(17), C(18), C(19), nullptr};
  const ColV P = TWO_D ? ColV{C(12), nullptr, nullptr, nullptr, nullptr, nullptr}
                       : ColV{C(20), nullptr, nullptr, nullptr, nullptr, nullptr};
  const StepCoef sc = sc_all[slot];
  const int nxm = g.nxm;
  const size_t pl = (size_t)j + (size_t)g.nym * i;
  const double tbp = nld<H>(t.tempbp + pl), ttp = nld<H>(t.temptp + pl);
  double rr[RPT][4];
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = ADJ ? RPT * tc + p : tc + TPC * p;
    if (k < nxm) {
      TE q0 = (TE)0, q1, q2, q3;
      const RowTab rt = (EARLY && p == 0) ? rte : row_tab<H>(t, k);
      const double u0 = uu[p][0], u1 = uu[p][1], u2 = uu[p][2], u3 = uu[p][3];
      // 2-D: vz(j-1,i+1) = vz(j-1), vy(j+1,i-1) = vy(j+1), pr(i-1) = pr
      const double zd = TWO_D ? Z.jm[k] : vv[p][0];
      const double yd = TWO_D ? Y.jp[k] : vv[p][1];
      const double pim = TWO_D ? P.c[k] : vv[p][3];
      // salinity buoyancy bycs * salc at this row, for the gravity component (SAL: salinity on)
      double sb = 0.0;
      if constexpr (SAL) sb = sbv[p];
      // all four right-hand sides from the staged columns before anything is stored
      const double sx = (EARLY && p == 0) ? rse[0] : ((k >= 1) ? tld<H>(TX + k - 1) : 0.0);
      const double sy = (EARLY && p == 0) ? rse[1] : tld<H>(TY + k);
      const double st = (EARLY && p == 0) ? rse[2] : tld<H>(TT + k);
      rr[p][0] = (k >= 1) ? rhs_vx<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, u0, q0, sb) * sx : 0.0;
      rr[p][1] = rhs_vy<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, zd, vv[p][2], u1, q1, sb) * sy;
      rr[p][2] = rhs_vz<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, yd, pim, u2, q2, sb) * sy;
      rr[p][3] = rhs_temp<TE, TWO_D, H>(g, rt, sc, k, X, Y, Z, T, tbp, ttp, u3, q3) * st;
      if (k >= 1) rux[c0 + k] = q0;
      ruy[c0 + k] = q1;
      ruz[c0 + k] = q2;
      rut[c0 + k] = q3;
    }
  }
  __syncthreads();  // the neighbour columns are dead from here on
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = ADJ ? RPT * tc + p : tc + TPC * p;
    if (k < nxm) {
      const int sk = (k % M) * LD + k / M;
      if (k >= 1) {
        const int r = k - 1;
        s_rhs[(r % M) * LD + r / M] = rr[p][0];
      }
      s_rhs[FLD + sk] = rr[p][1];
      s_rhs[2 * FLD + sk] = rr[p][2];
      s_rhs[3 * FLD + sk] = rr[p][3];
    }
  }
  // POL bit 4: each solving warp loads its field's forward-elimination factors before the
  // barrier below, so their latency overlaps the barrier and the other warps' stores
  constexpr bool PRE = (POL & 16) != 0 && (TPC / 32) == 4;
  CnFwd<M, H> fw;
  if constexpr (PRE) {
    const int warp = tc >> 5;
    fw.load((warp == 0) ? TX : ((warp == 3) ? TT : TY), tc & 31);
  }
  // identity padding rows: vx rows nxm-1 .. 32M-1, the others nxm .. 32M-1
  for (int r = nxm - 1 + tc; r < 32 * M; r += TPC) {
    const int sr = (r % M) * LD + r / M;
    s_rhs[sr] = 0.0;
    if (r >= nxm) {
      s_rhs[FLD + sr] = 0.0;
      s_rhs[2 * FLD + sr] = 0.0;
      s_rhs[3 * FLD + sr] = 0.0;
    }
  }
  __syncthreads();
  {
    const int warp = tc >> 5, lane = tc & 31;
    constexpr int NW = TPC / 32;
    for (int f = warp; f < 4; f += NW) {
      const double *Tb = (f == 0) ? TX : ((f == 3) ? TT : TY);
      if constexpr (PRE)
        cn_solve_chunk<M, LD, H, true>(s_rhs + f * FLD, Tb, lane, &fw);
      else
        cn_solve_chunk<M, LD, H>(s_rhs + f * FLD, Tb, lane);
    }
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = ADJ ? RPT * tc + p : tc + TPC * p;
    if (k < nxm) {
      const int sk = (k % M) * LD + k / M;
      if (k >= 1) {
        const int r = k - 1;
        vx_o[c0 + k] = X.c[k] + s_rhs[(r % M) * LD + r / M];
      } else {
        vx_o[c0] = 0.0;  // ImplicitAndUpdateVX.F90:86-87: vx(1) = vx(nx) = 0
        vx_o[c0 + nxm] = 0.0;
      }
      vy_o[c0 + k] = Y.c[k] + s_rhs[FLD + sk];
      vz_o[c0 + k] = Z.c[k] + s_rhs[2 * FLD + sk];
      temp_o[c0 + k] = T.c[k] + s_rhs[3 * FLD + sk];
    }
  }
}

// K1 on a tile of two neighbouring columns along y, (j0, i) and (j0 + 1, i), j0 even: a thread
// owns the same rows of both columns, so every metric coefficient it loads serves two cells, and
// warp f solves field f of both columns with one load of each CN factor (cn_solve_chunk2).  The
// staged set: vx, vy, vz, temp at j0 - 1 .. j0 + 2 (the y line) and at i +- 1 for both columns
// (in 3-D), and pr at both columns: 34 columns for two (17 a column instead of 21); in 2-D 18.
// The single-row operands left are vz(j0-1, i+1), vy(j0+2, i-1), pr(j0-1) and pr(i-1).
// Layout of the staged columns: centres F*2 + c (F = vx, vy, vz, temp; c = column 0, 1), the
// y-line ends 8 + F*2 + {0: j0-1, 1: j0+2}, then (3-D) z+ 16 + F*2 + c, z- 24 + F*2 + c, then pr.
constexpr int kK1Y2Cols = 34;
constexpr int kK1Y2Cols2D = 18;
__host__ __device__ inline size_t k1y2_smem(int M, bool two_d) {
  const int cs = k1_col_stride(M);
  const size_t st = (size_t)(two_d ? kK1Y2Cols2D : kK1Y2Cols) * cs * sizeof(double);
  const size_t rhs = (size_t)8 * cs * sizeof(double) + (size_t)8 * chunk_ld(M) * M * sizeof(double);
  return st > rhs ? st : rhs;
}

template <int M, int TPC, int RPT, typename TE, bool TWO_D, int CAP, bool SAL, int POL>
__global__ void __launch_bounds__(TPC, k1_min_blocks<CAP, TPC>())
    k_explicit_implicit_y2(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
                           const double *__restrict__ cn_tab, const double *__restrict__ vx,
                           const double *__restrict__ vy, const double *__restrict__ vz,
                           const double *__restrict__ temp, const double *__restrict__ pr,
                           TE *__restrict__ rux, TE *__restrict__ ruy, TE *__restrict__ ruz,
                           TE *__restrict__ rut, double *__restrict__ vx_o, double *__restrict__ vy_o,
                           double *__restrict__ vz_o, double *__restrict__ temp_o, int *__restrict__ err) {
  constexpr int LD = chunk_ld(M);
  constexpr int FLD = LD * M;
  constexpr int H = POL & 1;
  constexpr int NS = TWO_D ? kK1Y2Cols2D : kK1Y2Cols;
  constexpr int PRC = TWO_D ? 16 : 32;  // first pr column
  extern __shared__ __align__(128) unsigned char smem_k1[];
  __shared__ uint64_t bar;
  Geom g = g0;
  const int ldx = g.ldx;
  double *cols = reinterpret_cast<double *>(smem_k1);
  constexpr int CS = k1_col_stride(M);
  double *s_rhs = cols + (size_t)8 * CS;  // over the non-centre columns, after they are used
  const int tc = threadIdx.x;
  const int nyt = g.nym >> 1;
  const int j0 = 2 * (blockIdx.x % nyt), i = blockIdx.x / nyt;
  if (!inst_active(g, i)) {
    for (int c = 0; c < 2; ++c) {
      const size_t o = col_off(g, j0 + c, i);
      for (int k = tc; k < g.nx; k += TPC) temp_o[o + k] = temp[o + k];
    }
    return;
  }
  bind_instance(g, i);
  const int jm = wrap_dec(j0, g.nym), jp2 = wrap_inc(j0 + 1, g.nym);
  const int ip = zinc(g, i), im = zdec(g, i);
  size_t oc[2];
  oc[0] = col_off(g, j0, i);
  oc[1] = col_off(g, j0 + 1, i);
  if (tc == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tc == 0) {
    const uint32_t cb = (uint32_t)ldx * sizeof(double);
    mbar_arrive_expect_tx(&bar, (uint32_t)((size_t)NS * cb));
    const double *f4[4] = {vx, vy, vz, temp};
    const size_t ojm = col_off(g, jm, i), ojp2 = col_off(g, jp2, i);
#pragma unroll
    for (int F = 0; F < 4; ++F) {
      bulk_g2s(cols + (size_t)(F * 2 + 0) * CS, f4[F] + oc[0], cb, &bar);
      bulk_g2s(cols + (size_t)(F * 2 + 1) * CS, f4[F] + oc[1], cb, &bar);
      bulk_g2s(cols + (size_t)(8 + F * 2 + 0) * CS, f4[F] + ojm, cb, &bar);
      bulk_g2s(cols + (size_t)(8 + F * 2 + 1) * CS, f4[F] + ojp2, cb, &bar);
      if constexpr (!TWO_D) {
        bulk_g2s(cols + (size_t)(16 + F * 2 + 0) * CS, f4[F] + col_off(g, j0, ip), cb, &bar);
        bulk_g2s(cols + (size_t)(16 + F * 2 + 1) * CS, f4[F] + col_off(g, j0 + 1, ip), cb, &bar);
        bulk_g2s(cols + (size_t)(24 + F * 2 + 0) * CS, f4[F] + col_off(g, j0, im), cb, &bar);
        bulk_g2s(cols + (size_t)(24 + F * 2 + 1) * CS, f4[F] + col_off(g, j0 + 1, im), cb, &bar);
      }
    }
    bulk_g2s(cols + (size_t)(PRC + 0) * CS, pr + oc[0], cb, &bar);
    bulk_g2s(cols + (size_t)(PRC + 1) * CS, pr + oc[1], cb, &bar);
  }
  // single-row operands and the RK3 histories straight to registers, before the wait
  const size_t o_pjm = col_off(g, jm, i);                    // pr(j0 - 1)
  const size_t o_zd0 = col_off(g, jm, ip);                   // vz(j0 - 1, i + 1)
  const size_t o_yd1 = col_off(g, jp2, im);                  // vy(j0 + 2, i - 1)
  const size_t o_pim0 = col_off(g, j0, im), o_pim1 = col_off(g, j0 + 1, im);  // pr(., i - 1)
  double uu[RPT][2][4];
  double sv[RPT][5];  // {pr(j0-1), vz(j0-1,i+1), vy(j0+2,i-1), pr(j0,i-1), pr(j0+1,i-1)}
  double sbv[SAL ? RPT : 1][2];
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = tc + TPC * p;
    const bool in = k < g.nxm;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uu[p][c][0] = (in && k >= 1) ? sld<H>(rux + oc[c] + k) : 0.0;
      uu[p][c][1] = in ? sld<H>(ruy + oc[c] + k) : 0.0;
      uu[p][c][2] = in ? sld<H>(ruz + oc[c] + k) : 0.0;
      uu[p][c][3] = in ? sld<H>(rut + oc[c] + k) : 0.0;
      if constexpr (SAL) sbv[p][c] = in ? g.bycs * nld<H>(g.salc + oc[c] + k) : 0.0;
    }
    sv[p][0] = in ? nld<H>(pr + o_pjm + k) : 0.0;
    if constexpr (!TWO_D) {
      sv[p][1] = in ? nld<H>(vz + o_zd0 + k) : 0.0;
      sv[p][2] = in ? nld<H>(vy + o_yd1 + k) : 0.0;
      sv[p][3] = in ? nld<H>(pr + o_pim0 + k) : 0.0;
      sv[p][4] = in ? nld<H>(pr + o_pim1 + k) : 0.0;
    } else {
      sv[p][1] = sv[p][2] = sv[p][3] = sv[p][4] = 0.0;
    }
  }
  const int slot = sc_slot(g, i, ns);
  const size_t tsz = cn_table_size(M);
  const double *TX = cn_tab + (size_t)(slot * 3 + 0) * tsz;
  const double *TY = cn_tab + (size_t)(slot * 3 + 1) * tsz;
  const double *TT = cn_tab + (size_t)(slot * 3 + 2) * tsz;
  // POL bit 3: the first row's table operands and CN row scalings before the wait (as in
  // k_explicit_implicit); they serve both columns
  constexpr bool EARLY = (POL & 8) != 0;
  RowTab rte;
  double rse[3];
  if constexpr (EARLY) {
    if (tc < g.nxm) {
      rte = row_tab<H>(t, tc);
      rse[0] = (tc >= 1) ? tld<H>(TX + tc - 1) : 0.0;
      rse[1] = tld<H>(TY + tc);
      rse[2] = tld<H>(TT + tc);
    }
  }
  bool ok = mbar_wait(&bar, 0, kSpinLimit);
  if (g.wait_test_polls > 0) ok = ok && mbar_wait(&bar, 1, g.wait_test_polls);
  if (!__syncthreads_and(ok)) {
    if (tc == 0) atomicOr(err, 2);
    mbar_wait(&bar, 0, kDrainLimit);
    return;
  }
  auto C = [&](int q) { return (const double *)(cols + q * CS); };
  // column c of field F: {centre, j+1, j-1, i+1, i-1, -}
  auto colv = [&](int F, int c) {
    const double *ctr = C(F * 2 + c);
    const double *jpc = c == 0 ? C(F * 2 + 1) : C(8 + F * 2 + 1);
    const double *jmc = c == 0 ? C(8 + F * 2) : C(F * 2);
    if constexpr (TWO_D) return ColV{ctr, jpc, jmc, ctr, ctr, nullptr};
    return ColV{ctr, jpc, jmc, C(16 + F * 2 + c), C(24 + F * 2 + c), nullptr};
  };
  const StepCoef sc = sc_all[slot];
  const int nxm = g.nxm;
  double rr[RPT][2][4];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const ColV X = colv(0, c), Y = colv(1, c), Z = colv(2, c), T = colv(3, c);
    const ColV P{C(PRC + c), nullptr, nullptr, nullptr, nullptr, nullptr};
    const size_t pl = (size_t)(j0 + c) + (size_t)g.nym * i;
    const double tbp = nld<H>(t.tempbp + pl), ttp = nld<H>(t.temptp + pl);
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      if (k < nxm) {
        TE q0 = (TE)0, q1, q2, q3;
        const RowTab rt = (EARLY && p == 0) ? rte : row_tab<H>(t, k);
        // vz(j-1, i+1), vy(j+1, i-1), pr(j-1), pr(i-1) of column c
        double zd, yd, pjm, pim;
        if constexpr (TWO_D) {
          zd = c == 0 ? C(8 + 2 * 2)[k] : C(2 * 2)[k];        // vz(j-1)
          yd = c == 0 ? C(1 * 2 + 1)[k] : C(8 + 1 * 2 + 1)[k];  // vy(j+1)
          pim = P.c[k];
        } else {
          zd = c == 0 ? sv[p][1] : C(16 + 2 * 2 + 0)[k];        // vz(j0, i+1) staged for column 1
          yd = c == 0 ? C(24 + 1 * 2 + 1)[k] : sv[p][2];        // vy(j0+1, i-1) staged for column 0
          pim = c == 0 ? sv[p][3] : sv[p][4];
        }
        pjm = c == 0 ? sv[p][0] : C(PRC)[k];
        double sb = 0.0;
        if constexpr (SAL) sb = sbv[p][c];
        const double sx = (EARLY && p == 0) ? rse[0] : ((k >= 1) ? tld<H>(TX + k - 1) : 0.0);
        const double sy = (EARLY && p == 0) ? rse[1] : tld<H>(TY + k);
        const double st = (EARLY && p == 0) ? rse[2] : tld<H>(TT + k);
        rr[p][c][0] =
            (k >= 1) ? rhs_vx<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, uu[p][c][0], q0, sb) * sx : 0.0;
        rr[p][c][1] = rhs_vy<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, zd, pjm, uu[p][c][1], q1, sb) * sy;
        rr[p][c][2] = rhs_vz<TE, TWO_D, SAL, H>(g, rt, sc, k, X, Y, Z, T, P, yd, pim, uu[p][c][2], q2, sb) * sy;
        rr[p][c][3] = rhs_temp<TE, TWO_D, H>(g, rt, sc, k, X, Y, Z, T, tbp, ttp, uu[p][c][3], q3) * st;
        if (k >= 1) rux[oc[c] + k] = q0;
        ruy[oc[c] + k] = q1;
        ruz[oc[c] + k] = q2;
        rut[oc[c] + k] = q3;
      }
    }
  }
  __syncthreads();  // every non-centre column is dead from here on
  // system s = c * 4 + F over the dead columns; padding rows as in the one-column kernel
#pragma unroll
  for (int p = 0; p < RPT; ++p) {
    const int k = tc + TPC * p;
    if (k < nxm) {
      const int sk = (k % M) * LD + k / M;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        double *sr = s_rhs + (size_t)c * 4 * FLD;
        if (k >= 1) {
          const int r = k - 1;
          sr[(r % M) * LD + r / M] = rr[p][c][0];
        }
        sr[FLD + sk] = rr[p][c][1];
        sr[2 * FLD + sk] = rr[p][c][2];
        sr[3 * FLD + sk] = rr[p][c][3];
      }
    }
  }
  for (int r = nxm - 1 + tc; r < 32 * M; r += TPC) {
    const int sr = (r % M) * LD + r / M;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double *b = s_rhs + (size_t)c * 4 * FLD;
      b[sr] = 0.0;
      if (r >= nxm) {
        b[FLD + sr] = 0.0;
        b[2 * FLD + sr] = 0.0;
        b[3 * FLD + sr] = 0.0;
      }
    }
  }
  __syncthreads();
  {
    const int warp = tc >> 5, lane = tc & 31;
    constexpr int NW = TPC / 32;
    if constexpr (NW >= 8) {  // a warp per system: no warp idles through the solves
      for (int sidx = warp; sidx < 8; sidx += NW) {
        const int f = sidx & 3;
        const double *Tb = (f == 0) ? TX : ((f == 3) ? TT : TY);
        cn_solve_chunk<M, LD, H>(s_rhs + (size_t)((sidx >> 2) * 4 + f) * FLD, Tb, lane);
      }
    } else {  // fewer warps: a warp per field, both columns with one load of each factor
      for (int f = warp; f < 4; f += NW) {
        const double *Tb = (f == 0) ? TX : ((f == 3) ? TT : TY);
        cn_solve_chunk2<M, LD, H>(s_rhs + f * FLD, s_rhs + (4 + f) * FLD, Tb, lane);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double *sr = s_rhs + (size_t)c * 4 * FLD;
    const double *Xc = C(0 * 2 + c), *Yc = C(1 * 2 + c), *Zc = C(2 * 2 + c), *Tc = C(3 * 2 + c);
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      if (k < nxm) {
        const int sk = (k % M) * LD + k / M;
        if (k >= 1) {
          const int r = k - 1;
          vx_o[oc[c] + k] = Xc[k] + sr[(r % M) * LD + r / M];
        } else {
          vx_o[oc[c]] = 0.0;  // ImplicitAndUpdateVX.F90:86-87: vx(1) = vx(nx) = 0
          vx_o[oc[c] + nxm] = 0.0;
        }
        vy_o[oc[c] + k] = Yc[k] + sr[FLD + sk];
        vz_o[oc[c] + k] = Zc[k] + sr[2 * FLD + sk];
        temp_o[oc[c] + k] = Tc[k] + sr[3 * FLD + sk];
      }
    }
  }
}

// The two-column tile: ncol / 2 blocks; needs an even nym (every x-column pair within a row of
// the y-z plane) and an even ncol.
template <int M, int TPC, int RPT, typename TE, bool TWO_D, int CAP, bool SAL, int POL>
cudaError_t launch_k1y2_cfg(const LaunchCtx &L, const SubstepBuffers &b, int ns, int ncol) {
  if ((L.g.nym & 1) || (ncol & 1)) return cudaErrorInvalidValue;
  const size_t smem = k1y2_smem(M, TWO_D);
  auto kern = k_explicit_implicit_y2<M, TPC, RPT, TE, TWO_D, CAP, SAL, POL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<ncol / 2, TPC, smem, L.stream>>>(L.g, L.t, b.sc, ns, b.cn_tab, b.vx, b.vy, b.vz, b.temp, b.pr,
                                          (TE *)b.rux, (TE *)b.ruy, (TE *)b.ruz, (TE *)b.rut, b.vx_o, b.vy_o,
                                          b.vz_o, b.temp_o, b.err);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// K1, persistent form: one block per SM, G groups of TPC threads.  The block stages the tables
// every column reads (the 12 metric arrays and the substep's three CN factor sets) into shared
// memory once, then each group works through columns blockIdx.x*G + grp, + gridDim.x*G, ... with
// its own staging slot and mbarrier, exactly as the one-column kernel does per block; table
// reads are shared-memory loads instead of L1/L2 hits.  Groups synchronise on named barriers
// (id 1 + grp) and never wait for one another.  Single domains only (a batch has CN tables per
// instance).
// ------------------------------------------------------------------------------------------
__host__ __device__ constexpr int k1p_cn_doubles(int M) { return 192 * M + 576; }
__host__ __device__ constexpr size_t k1p_slot_doubles(int M, bool two_d) {
  const size_t st = (size_t)(two_d ? kK1StateCols2D : kK1StateCols) * k1_col_stride(M);
  const size_t rhs = (size_t)kK1Centre * k1_col_stride(M) + (size_t)4 * chunk_ld(M) * M;
  const size_t d = st > rhs ? st : rhs;
  return (d + 15) / 16 * 16;  // 128-byte aligned slots
}
__host__ __device__ constexpr size_t k1p_table_doubles(int M) {
  return (size_t)12 * k1_col_stride(M) + (size_t)3 * k1p_cn_doubles(M);
}
// Groups per block: as many staging slots as fit beside the tables in 227 KB, at most 4.
__host__ __device__ constexpr int k1p_groups(int M, bool two_d) {
  const size_t avail = (size_t)232448 - 512 - k1p_table_doubles(M) * 8;
  const size_t g = avail / (k1p_slot_doubles(M, two_d) * 8);
  return g > 4 ? 4 : (int)g;
}
__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ bool group_and(int id, int nthreads, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int M, int TPC, int RPT, typename TE, bool TWO_D, bool SAL, int G>
__global__ void __launch_bounds__(TPC * G, 1)
    k_explicit_implicit_p(Geom g0, Tables t, const StepCoef *__restrict__ sc_all, int ns,
                          const double *__restrict__ cn_tab, const double *__restrict__ vx,
                          const double *__restrict__ vy, const double *__restrict__ vz,
                          const double *__restrict__ temp, const double *__restrict__ pr,
                          TE *__restrict__ rux, TE *__restrict__ ruy, TE *__restrict__ ruz,
                          TE *__restrict__ rut, double *__restrict__ vx_o, double *__restrict__ vy_o,
                          double *__restrict__ vz_o, double *__restrict__ temp_o, int *__restrict__ err,
                          int ncol) {
  constexpr int LD = chunk_ld(M);
  constexpr int FLD = LD * M;
  constexpr int CS = k1_col_stride(M);
  constexpr int TSZ = k1p_cn_doubles(M);
  constexpr size_t SLOT = k1p_slot_doubles(M, TWO_D);
  constexpr int NT = TPC * G;
  extern __shared__ __align__(128) unsigned char smem_k1p[];
  __shared__ uint64_t tbar, bars[G];
  double *tm = reinterpret_cast<double *>(smem_k1p);  // 12 metric arrays at stride CS
  double *tcn = tm + 12 * CS;                          // CN factors of vx, vy/vz, temp
  const int tid = threadIdx.x, grp = tid / TPC, tc = tid % TPC;
  const int slot = ns;  // single domain: one table set per substep
  if (tid == 0) {
    mbar_init(&tbar, 1);
#pragma unroll
    for (int q = 0; q < G; ++q) mbar_init(&bars[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t mb = (uint32_t)(((g0.nx + 1) & ~1) * sizeof(double));  // rows rounded to 16 bytes
    mbar_arrive_expect_tx(&tbar, 12 * mb + 3 * (uint32_t)TSZ * (uint32_t)sizeof(double));
    const double *src[12] = {t.idx,   t.udx3c, t.udx3m, t.ap3ck,  t.ac3ck,  t.am3ck,
                             t.ap3sk, t.ac3sk, t.am3sk, t.ap3ssk, t.ac3ssk, t.am3ssk};
#pragma unroll
    for (int q = 0; q < 12; ++q) bulk_g2s(tm + (size_t)q * CS, src[q], mb, &tbar);
#pragma unroll
    for (int m = 0; m < 3; ++m)
      bulk_g2s(tcn + (size_t)m * TSZ, cn_tab + (size_t)(slot * 3 + m) * TSZ, (uint32_t)TSZ * sizeof(double), &tbar);
  }
  const bool tok = mbar_wait(&tbar, 0, kSpinLimit);
  if (!__syncthreads_and(tok)) {
    if (tid == 0) atomicOr(err, 2);
    mbar_wait(&tbar, 0, kDrainLimit);
    return;
  }
  Tables ts = t;  // the metric arrays from shared memory
  ts.idx = tm;
  ts.udx3c = tm + CS;
  ts.udx3m = tm + 2 * CS;
  ts.ap3ck = tm + 3 * CS;
  ts.ac3ck = tm + 4 * CS;
  ts.am3ck = tm + 5 * CS;
  ts.ap3sk = tm + 6 * CS;
  ts.ac3sk = tm + 7 * CS;
  ts.am3sk = tm + 8 * CS;
  ts.ap3ssk = tm + 9 * CS;
  ts.ac3ssk = tm + 10 * CS;
  ts.am3ssk = tm + 11 * CS;
  const double *TX = tcn, *TY = tcn + TSZ, *TT = tcn + 2 * TSZ;
  const StepCoef sc = sc_all[slot];
  double *cols = tcn + 3 * TSZ + (size_t)grp * SLOT;
  double *s_rhs = cols + (size_t)kK1Centre * CS;
  uint64_t *bar = &bars[grp];
  const int gid = 1 + grp;
  const int ldx = g0.ldx, nxm = g0.nxm;
  uint32_t ph = 0;
  for (int colid = blockIdx.x * G + grp; colid < ncol; colid += gridDim.x * G) {
    Geom g = g0;
    const int j = colid % g.nym, i = colid / g.nym;
    const size_t c0 = col_off(g, j, i);
    if (!inst_active(g, i)) {
      for (int k = tc; k < g.nx; k += TPC) temp_o[c0 + k] = temp[c0 + k];
      continue;
    }
    const int jp = wrap_inc(j, g.nym), jm = wrap_dec(j, g.nym);
    const int ip = zinc(g, i), im = zdec(g, i);
    if (tc == 0) {
      const size_t oc = c0, ojp = col_off(g, jp, i), ojm = col_off(g, jm, i), oip = col_off(g, j, ip),
                   oim = col_off(g, j, im);
      const uint32_t cb = (uint32_t)ldx * sizeof(double);
      mbar_arrive_expect_tx(bar, (uint32_t)k1_stage_bytes(ldx, TWO_D));
      if constexpr (TWO_D) {
        const double *src[kK1StateCols2D] = {vx + oc,   vy + oc,    vz + oc, temp + oc, vx + ojp, vx + ojm, vy + ojp,
                                             vy + ojm,  vz + ojp,   vz + ojm, temp + ojp, temp + ojm, pr + oc};
#pragma unroll
        for (int q = 0; q < kK1StateCols2D; ++q) bulk_g2s(cols + (size_t)q * CS, src[q], cb, bar);
      } else {
        const double *src[kK1StateCols] = {vx + oc,    vy + oc,    vz + oc,    temp + oc,  vx + ojp,   vx + ojm,
                                           vx + oip,   vx + oim,   vy + ojp,   vy + ojm,   vy + oip,   vy + oim,
                                           vz + ojp,   vz + ojm,   vz + oip,   vz + oim,   temp + ojp, temp + ojm,
                                           temp + oip, temp + oim, pr + oc};
#pragma unroll
        for (int q = 0; q < kK1StateCols; ++q) bulk_g2s(cols + (size_t)q * CS, src[q], cb, bar);
      }
    }
    const size_t o_jm = col_off(g, jm, i), o_im = col_off(g, j, im);
    const size_t o_jpim = col_off(g, jp, im), o_jmip = col_off(g, jm, ip);
    double uu[RPT][4], vv[RPT][4];
    double sbv[SAL ? RPT : 1];
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      const bool in = k < nxm;
      uu[p][0] = (in && k >= 1) ? sld<1>(rux + c0 + k) : 0.0;
      uu[p][1] = in ? sld<1>(ruy + c0 + k) : 0.0;
      uu[p][2] = in ? sld<1>(ruz + c0 + k) : 0.0;
      uu[p][3] = in ? sld<1>(rut + c0 + k) : 0.0;
      if constexpr (TWO_D) {
        vv[p][0] = vv[p][1] = vv[p][3] = 0.0;
      } else {
        vv[p][0] = in ? nld<1>(vz + o_jmip + k) : 0.0;
        vv[p][1] = in ? nld<1>(vy + o_jpim + k) : 0.0;
        vv[p][3] = in ? nld<1>(pr + o_im + k) : 0.0;
      }
      vv[p][2] = in ? nld<1>(pr + o_jm + k) : 0.0;
      if constexpr (SAL) sbv[p] = in ? g.bycs * nld<1>(g.salc + c0 + k) : 0.0;
    }
    bool ok = mbar_wait(bar, ph & 1, kSpinLimit);
    if (g.wait_test_polls > 0) ok = ok && mbar_wait(bar, (ph & 1) ^ 1, g.wait_test_polls);
    if (!group_and(gid, TPC, ok)) {
      if (tc == 0) atomicOr(err, 2);
      mbar_wait(bar, ph & 1, kDrainLimit);
      break;  // the whole group leaves; the other groups are not affected
    }
    ++ph;
    auto C = [&](int q) { return (const double *)(cols + q * CS); };
    const ColV X = TWO_D ? ColV{C(0), C(4), C(5), C(0), C(0), nullptr} : ColV{C(0), C(4), C(5), C(6), C(7), nullptr};
    const ColV Y = TWO_D ? ColV{C(1), C(6), C(7), C(1), C(1), nullptr} : ColV{C(1), C(8), C(9), C(10), C(11), nullptr};
    const ColV Z = TWO_D ? ColV{C(2), C(8), C(9), C(2), C(2), nullptr} : ColV{C(2), C(12), C(13), C(14), C(15), nullptr};
    const ColV T = TWO_D ? ColV{C(3), C(10), C(11), C(3), C(3), nullptr} : ColV{C(3), C(16), C(17), C(18), C(19), nullptr};
    const ColV P = TWO_D ? ColV{C(12), nullptr, nullptr, nullptr, nullptr, nullptr}
                         : ColV{C(20), nullptr, nullptr, nullptr, nullptr, nullptr};
    const size_t pl = (size_t)j + (size_t)g.nym * i;
    const double tbp = nld<1>(t.tempbp + pl), ttp = nld<1>(t.temptp + pl);
    double rr[RPT][4];
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      if (k < nxm) {
        TE q0 = (TE)0, q1, q2, q3;
        const RowTab rt = row_tab<2>(ts, k);
        const double zd = TWO_D ? Z.jm[k] : vv[p][0];
        const double yd = TWO_D ? Y.jp[k] : vv[p][1];
        const double pim = TWO_D ? P.c[k] : vv[p][3];
        double sb = 0.0;
        if constexpr (SAL) sb = sbv[p];
        rr[p][0] = (k >= 1) ? rhs_vx<TE, TWO_D, SAL, 2>(g, rt, sc, k, X, Y, Z, T, P, uu[p][0], q0, sb) * TX[k - 1] : 0.0;
        rr[p][1] = rhs_vy<TE, TWO_D, SAL, 2>(g, rt, sc, k, X, Y, Z, T, P, zd, vv[p][2], uu[p][1], q1, sb) * TY[k];
        rr[p][2] = rhs_vz<TE, TWO_D, SAL, 2>(g, rt, sc, k, X, Y, Z, T, P, yd, pim, uu[p][2], q2, sb) * TY[k];
        rr[p][3] = rhs_temp<TE, TWO_D, 2>(g, rt, sc, k, X, Y, Z, T, tbp, ttp, uu[p][3], q3) * TT[k];
        if (k >= 1) rux[c0 + k] = q0;
        ruy[c0 + k] = q1;
        ruz[c0 + k] = q2;
        rut[c0 + k] = q3;
      }
    }
    group_sync(gid, TPC);  // the neighbour columns are dead from here on
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      if (k < nxm) {
        const int sk = (k % M) * LD + k / M;
        if (k >= 1) {
          const int r = k - 1;
          s_rhs[(r % M) * LD + r / M] = rr[p][0];
        }
        s_rhs[FLD + sk] = rr[p][1];
        s_rhs[2 * FLD + sk] = rr[p][2];
        s_rhs[3 * FLD + sk] = rr[p][3];
      }
    }
    for (int r = nxm - 1 + tc; r < 32 * M; r += TPC) {
      const int sr = (r % M) * LD + r / M;
      s_rhs[sr] = 0.0;
      if (r >= nxm) {
        s_rhs[FLD + sr] = 0.0;
        s_rhs[2 * FLD + sr] = 0.0;
        s_rhs[3 * FLD + sr] = 0.0;
      }
    }
    group_sync(gid, TPC);
    {
      const int warp = tc >> 5, lane = tc & 31;
      constexpr int NW = TPC / 32;
      for (int f = warp; f < 4; f += NW) {
        const double *Tb = (f == 0) ? TX : ((f == 3) ? TT : TY);
        cn_solve_chunk<M, LD, 2>(s_rhs + f * FLD, Tb, lane);
      }
    }
    group_sync(gid, TPC);
#pragma unroll
    for (int p = 0; p < RPT; ++p) {
      const int k = tc + TPC * p;
      if (k < nxm) {
        const int sk = (k % M) * LD + k / M;
        if (k >= 1) {
          const int r = k - 1;
          vx_o[c0 + k] = X.c[k] + s_rhs[(r % M) * LD + r / M];
        } else {
          vx_o[c0] = 0.0;  // ImplicitAndUpdateVX.F90:86-87: vx(1) = vx(nx) = 0
          vx_o[c0 + nxm] = 0.0;
        }
        vy_o[c0 + k] = Y.c[k] + s_rhs[FLD + sk];
        vz_o[c0 + k] = Z.c[k] + s_rhs[2 * FLD + sk];
        temp_o[c0 + k] = T.c[k] + s_rhs[3 * FLD + sk];
      }
    }
    // the slot is rewritten by the next column's bulk copies (async proxy): order this group's
    // shared-memory reads and writes before them
    fence_proxy_async_smem();
    group_sync(gid, TPC);
  }
  (void)NT;
}

template <int M, int TPC, int RPT, typename TE, bool TWO_D, bool SAL>
cudaError_t launch_k1p_cfg(const LaunchCtx &L, const SubstepBuffers &b, int ns, int ncol) {
  constexpr int G = k1p_groups(M, TWO_D);
  if constexpr (G < 2) {
    return cudaErrorInvalidValue;  // the tables leave room for fewer than two groups
  } else {
    if (L.g.batch) return cudaErrorInvalidValue;  // CN tables per instance
    static int nsm = 0;
    if (nsm == 0) {
      int dev = 0;
      cudaGetDevice(&dev);
      if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
    }
    const size_t smem = (k1p_table_doubles(M) + (size_t)G * k1p_slot_doubles(M, TWO_D)) * sizeof(double);
    auto kern = k_explicit_implicit_p<M, TPC, RPT, TE, TWO_D, SAL, G>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = std::min(nsm, (ncol + G - 1) / G);
    kern<<<grid, TPC * G, smem, L.stream>>>(L.g, L.t, b.sc, ns, b.cn_tab, b.vx, b.vy, b.vz, b.temp, b.pr,
                                            (TE *)b.rux, (TE *)b.ruy, (TE *)b.ruz, (TE *)b.rut, b.vx_o, b.vy_o,
                                            b.vz_o, b.temp_o, b.err, ncol);
    return cudaGetLastError();
  }
}

template <int M, int TPC, int RPT, typename TE, bool TWO_D, int CAP, bool SAL, int POL>
cudaError_t launch_k1_cfg(const LaunchCtx &L, const SubstepBuffers &b, int ns, int ncol) {
  const size_t smem = k1_smem(L.g.ldx, M, TWO_D);
  auto kern = k_explicit_implicit<M, TPC, RPT, TE, TWO_D, CAP, SAL, POL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<ncol, TPC, smem, L.stream>>>(L.g, L.t, b.sc, ns, b.cn_tab, b.vx, b.vy, b.vz, b.temp, b.pr,
                                      (TE *)b.rux, (TE *)b.ruy, (TE *)b.ruz, (TE *)b.rut, b.vx_o, b.vy_o,
                                      b.vz_o, b.temp_o, b.err);
  return cudaGetLastError();
}

// Launch shapes of K1 per M = {1, 2, 4, 8, 12, 16, 24, 32} (rows per lane of the CN solves):
// {threads per column, rows per thread, register cap level, policy (bit 0: the cache hints of
// tld / nld / sld; bit 1: tables in shared memory; bit 2: adjacent rows per thread; bit 3: the
// row operands loaded before the staging wait; bit 4: the solves' forward factors loaded before
// the barrier that precedes the solves), columns per
// block along y (1, or 2 for the tile of k_explicit_implicit_y2; 0 for the persistent
// k_explicit_implicit_p with its groups of `threads` threads)}, threads x rows >= 32 M.  The
// first entry is the default.
struct K1Shape {
  int tpc, rpt, cap, pol, ny;
};
constexpr int kK1MaxShapes = 8;
constexpr int k1_m_index(int M) {
  return M == 1 ? 0 : M == 2 ? 1 : M == 4 ? 2 : M == 8 ? 3 : M == 12 ? 4 : M == 16 ? 5 : M == 24 ? 6 : 7;
}
constexpr int kK1ShapeCount[8] = {1, 5, 8, 8, 8, 8, 6, 5};
constexpr K1Shape kK1Shapes[8][kK1MaxShapes] = {
    {{32, 1, 0, 0, 1}},                                                                  // M = 1   (nxm <= 32)
    {{64, 1, 0, 0, 1}, {32, 2, 1, 0, 1}, {64, 1, 0, 1, 1}, {64, 1, 0, 1, 2}, {64, 1, 0, 9, 2}},  // M = 2
    {{128, 1, 0, 0, 1}, {64, 2, 1, 0, 1}, {128, 1, 2, 0, 1}, {128, 1, 0, 1, 1},           // M = 4   (<= 128)
     {128, 1, 1, 1, 2}, {128, 1, 0, 1, 2}, {128, 1, 0, 2, 0}, {128, 1, 1, 9, 2}},
    {{128, 2, 1, 0, 1}, {128, 2, 1, 25, 1}, {128, 2, 1, 1, 1}, {128, 2, 1, 9, 2},         // M = 8   (<= 256)
     {128, 2, 1, 9, 1}, {256, 1, 1, 1, 2}, {128, 2, 1, 1, 2}, {128, 2, 0, 2, 0}},
    {{128, 3, 1, 0, 1}, {128, 3, 1, 9, 1}, {128, 3, 0, 9, 1}, {128, 3, 0, 0, 1},          // M = 12  (<= 384)
     {384, 1, 2, 0, 1}, {384, 1, 0, 1, 1}, {128, 3, 1, 1, 1}, {384, 1, 0, 1, 2}},
    {{128, 4, 1, 0, 1}, {256, 2, 1, 0, 1}, {128, 4, 1, 9, 1}, {128, 4, 0, 0, 1},          // M = 16  (<= 512)
     {512, 1, 2, 0, 1}, {128, 4, 1, 1, 1}, {128, 4, 1, 8, 1}, {128, 4, 1, 24, 1}},
    {{256, 3, 1, 0, 1}, {384, 2, 0, 0, 1}, {256, 4, 1, 0, 1}, {256, 3, 1, 1, 1},          // M = 24  (<= 768)
     {384, 2, 0, 1, 1}, {384, 2, 0, 1, 2}},
    {{256, 4, 1, 0, 1}, {512, 2, 0, 0, 1}, {256, 4, 1, 1, 1}, {512, 2, 0, 1, 1},          // M = 32  (<= 1024)
     {512, 2, 0, 1, 2}},
};

template <int M, int V, typename TE, bool TWO_D, bool SAL>
cudaError_t launch_k1_v(const LaunchCtx &L, const SubstepBuffers &b, int ns, int ncol) {
  constexpr int mi = k1_m_index(M);
  if constexpr (V < kK1ShapeCount[mi]) {
    constexpr int TPC = kK1Shapes[mi][V].tpc, RPT = kK1Shapes[mi][V].rpt;
    constexpr int CAP = kK1Shapes[mi][V].cap, POL = kK1Shapes[mi][V].pol;
    static_assert(TPC * RPT >= 32 * M, "K1 shape must cover 32*M rows");
    if constexpr (kK1Shapes[mi][V].ny == 2)
      return launch_k1y2_cfg<M, TPC, RPT, TE, TWO_D, CAP, SAL, POL>(L, b, ns, ncol);
    else if constexpr (kK1Shapes[mi][V].ny == 0)
      return launch_k1p_cfg<M, TPC, RPT, TE, TWO_D, SAL>(L, b, ns, ncol);
    else
      return launch_k1_cfg<M, TPC, RPT, TE, TWO_D, CAP, SAL, POL>(L, b, ns, ncol);
  } else {
    return cudaErrorInvalidValue;
  }
}

template <int M, typename TE, bool TWO_D, bool SAL>
cudaError_t launch_k1_M(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  switch (var) {
    case 0: return launch_k1_v<M, 0, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 1: return launch_k1_v<M, 1, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 2: return launch_k1_v<M, 2, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 3: return launch_k1_v<M, 3, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 4: return launch_k1_v<M, 4, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 5: return launch_k1_v<M, 5, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 6: return launch_k1_v<M, 6, TE, TWO_D, SAL>(L, b, ns, ncol);
    case 7: return launch_k1_v<M, 7, TE, TWO_D, SAL>(L, b, ns, ncol);
  }
  return cudaErrorInvalidValue;
}

template <typename TE, bool TWO_D, bool SAL>
cudaError_t launch_k1_T(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  switch (L.M) {
    case 1: return launch_k1_M<1, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 2: return launch_k1_M<2, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 4: return launch_k1_M<4, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 8: return launch_k1_M<8, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 12: return launch_k1_M<12, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 16: return launch_k1_M<16, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 24: return launch_k1_M<24, TE, TWO_D, SAL>(L, b, ns, var, ncol);
    case 32: return launch_k1_M<32, TE, TWO_D, SAL>(L, b, ns, var, ncol);
  }
  return cudaErrorInvalidValue;
}

}  // namespace afid
