// afid_device.cuh — device-side building blocks shared by the substep kernels.
//
// Layout in HBM (one context = one domain): every 3-D field is x-fastest like the reference's
// Fortran arrays (param.F90:100-108) without halos: element (k, j, i) (0-based) sits at
// k + ldx * (j + nym * i) with ldx >= nx = nxm + 1 padded to a multiple of 8 elements so that
// each x-column starts on a 64-byte boundary.  Periodic y/z neighbours are reached by index
// wrap instead of the reference's halo copies (update_halo, halo_common.F90:43-109).
// The Poisson spectrum is complex, x-fastest: (k, ky, i|kz) at k + ldxc * (ky + nyh * i),
// nyh = nym/2 + 1 — the reference's dphc / cz1 arrays (pressure.F90:120-134) in one layout.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace afid {

constexpr int kWarp = 32;
constexpr int kMaxFftPasses = 24;

struct Geom {
  int nxm, nym, nzm, nx;
  int ldx;    // x stride of real fields (elements)
  int nyh;    // nym/2 + 1
  int ldxc;   // x stride of the complex spectrum (elements)
  double dx, dy, dz, dyq, dzq;
  double ren, pect, byct, gy;
  double rren, rpect;                 // 1/ren, 1/pect
  double udyq_re, udzq_re, udyq_pe, udzq_pe;  // dyq/ren, dzq/ren, dyq/pect, dzq/pect
  double xplusu, xminusu;
  int active_t, gaxis, inslws, inslwn, tfixs, tfixn;
  // Batch mode (batch != 0): the z index numbers independent 2-D instances of one size class;
  // they do not couple along z and each has its own scalars, RK3 coefficients, CN tables,
  // wavenumbers and an active flag.
  int batch;
  const struct InstScal *inst;   // [nzm] per-instance scalars (batch mode), else nullptr
  const unsigned char *active;   // [nzm] 1 = advance this instance (batch mode), else nullptr
  // Salinity buoyancy (AddSalBuoyancy, salinity.F90:494-506): the forcing along gaxis loses
  // bycs * salc at rows 0..nxm-1; nullptr when no active salinity is coupled.
  const double *salc;
  double bycs;
  // Test hook of the bounded waits (afid_gpu_set_wait_test): when non-zero, the staging waits of
  // K1 and of the tensor-copy transforms also wait for an mbarrier phase that nothing
  // completes, for at most this many polls, so the timeout path runs; 0 in normal operation.
  long long wait_test_polls;
};

// Shared-memory stride of the chunked tridiagonal layout (row r of a 32-chunk system at
// (r % M) * LD + r / M, chunk q of lane l at q * LD + l): the smallest stride >= 32 that makes
// the row-ordered accesses of a half-warp hit distinct 8-byte banks (2-way for M = 12, 24).
__host__ __device__ constexpr int chunk_ld(int M) {
  return M == 1 ? 32 : M == 2 ? 40 : M == 4 ? 36 : M == 8 ? 34 : 33;
}

// Scalars that differ between the instances of a batch (aspect ratio, Ra, Pr).
struct InstScal {
  double dy, dyq, ren, pect, rren, rpect, udyq_re, udyq_pe;
};

// Device-resident per-substep scalars (written by the coefficient kernel, read by every
// kernel of the substep, so a captured step graph does not depend on dt).
struct StepCoef {
  double al, ga, ro, dt, beta;
  double alre, alpec;  // al/ren (ImplicitAndUpdateVX.F90:26), al/pect (ImplicitAndUpdateTemp.F90:22)
};

// 1-D metric tables on the device (0-based copies of the reference's arrays).
struct Tables {
  const double *udx3c, *udx3m, *idx;  // idx = 1/udx3m (ExplicitTermsVX.F90:30-32)
  const double *ap3ck, *ac3ck, *am3ck;
  const double *ap3sk, *ac3sk, *am3sk;
  const double *ap3ssk, *ac3ssk, *am3ssk;
  const double *amphk, *acphk, *apphk;
  const double *ak1, *ak2;
  const double *g3rc;
  const double *g3rm;  // cell-centre metric (CreateGrid.F90), for the profile gradients
  const double *tempbp, *temptp;  // nym*nzm, y fastest
};

struct FftPlan {
  int n;
  int npass;
  int radix[kMaxFftPasses];
};

__device__ __forceinline__ int wrap_inc(int a, int n) { return (a + 1 == n) ? 0 : a + 1; }
__device__ __forceinline__ int wrap_dec(int a, int n) { return (a == 0) ? n - 1 : a - 1; }

// z neighbours: periodic for one domain, the instance itself in batch mode (2-D instances).
__device__ __forceinline__ int zinc(const Geom &g, int i) { return g.batch ? i : wrap_inc(i, g.nzm); }
__device__ __forceinline__ int zdec(const Geom &g, int i) { return g.batch ? i : wrap_dec(i, g.nzm); }
// Batch mode: active[i] per instance (i = z index).  A single 3-D domain with step control on
// the device uses active[0] for the whole domain.
__device__ __forceinline__ bool inst_active(const Geom &g, int i) {
  return !g.active || g.active[g.batch ? i : 0] != 0;
}
// Load the scalars of instance i into a block-local copy of the geometry (batch mode).
__device__ __forceinline__ void bind_instance(Geom &g, int i) {
  if (g.inst) {
    const InstScal s = g.inst[i];
    g.dy = s.dy;
    g.dyq = s.dyq;
    g.ren = s.ren;
    g.pect = s.pect;
    g.rren = s.rren;
    g.rpect = s.rpect;
    g.udyq_re = s.udyq_re;
    g.udyq_pe = s.udyq_pe;
  }
}
// Index of the RK3 coefficients of substep ns (per instance in batch mode).
__device__ __forceinline__ int sc_slot(const Geom &g, int i, int ns) { return (g.batch ? 3 * i : 0) + ns; }
// z extent that the FFT normalisation 1/(nym*nzm) uses.
__device__ __forceinline__ double nz_norm(const Geom &g) { return g.batch ? 1.0 : (double)g.nzm; }

__device__ __forceinline__ size_t col_off(const Geom &g, int j, int i) {
  return (size_t)(j + (size_t)g.nym * i) * (size_t)g.ldx;
}

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  C r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_mi(C a) {
  C r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

// ------------------------------------------------------------------------------------------
// Shared-memory Stockham FFT (auto-sort), radices 2, 3, 4, 5, batch of B sequences of length
// N stored contiguously (seq s at buf[s*N]).  Forward uses exp(-2 pi i m/N) twiddles from the
// table tw[m] = (cos(2 pi m/N), -sin(2 pi m/N)); the inverse conjugates them and is
// unnormalised, the FFTW_BACKWARD convention the reference uses (pressure.F90:189,193).
// Pass p with radix R and Ns = product of earlier radices reads x[j + q*N/R] and writes
// y[(j/Ns)*Ns*R + (j%Ns) + q*Ns] after twiddling input q by w^(q*(j%Ns)*N/(Ns*R)).
// Returns the buffer holding the result.  All threads of the block must call it.
// ------------------------------------------------------------------------------------------
template <bool INV, typename T>
__device__ typename Cplx<T>::type *fft_block(typename Cplx<T>::type *buf0,
                                             typename Cplx<T>::type *buf1, int B,
                                             const FftPlan &pl,
                                             const typename Cplx<T>::type *__restrict__ tw) {
  using C = typename Cplx<T>::type;
  const int N = pl.n;
  C *in = buf0, *out = buf1;
  int Ns = 1;
  for (int p = 0; p < pl.npass; ++p) {
    const int R = pl.radix[p];
    const int NR = N / R;
    const int tstride = N / (Ns * R);
    const int total = B * NR;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int s = b / NR;
      const int jj = b - s * NR;
      const int k = jj % Ns;
      const C *src = in + (size_t)s * N + jj;
      C *dst = out + (size_t)s * N + (jj / Ns) * Ns * R + k;
      C a[5];
#pragma unroll
      for (int q = 0; q < 5; ++q)
        if (q < R) a[q] = src[q * NR];
      if (Ns > 1) {
#pragma unroll
        for (int q = 1; q < 5; ++q) {
          if (q < R) {
            C w = tw[q * k * tstride];
            if (INV) w.y = -w.y;
            a[q] = cmul(a[q], w);
          }
        }
      }
      if (R == 2) {
        dst[0] = cadd(a[0], a[1]);
        dst[Ns] = csub(a[0], a[1]);
      } else if (R == 4) {
        C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        C t2 = cadd(a[1], a[3]), t3 = mul_mi<INV>(csub(a[1], a[3]));
        dst[0] = cadd(t0, t2);
        dst[Ns] = cadd(t1, t3);
        dst[2 * Ns] = csub(t0, t2);
        dst[3 * Ns] = csub(t1, t3);
      } else if (R == 3) {
        // y1,2 = a0 - (a1+a2)/2 -/+ i (sqrt(3)/2)(a1-a2) for the forward sign
        const T s3 = (T)0.86602540378443864676;  // sqrt(3)/2
        C t1 = cadd(a[1], a[2]);
        C t2;
        t2.x = a[0].x - (T)0.5 * t1.x;
        t2.y = a[0].y - (T)0.5 * t1.y;
        C d = csub(a[1], a[2]);
        C t3 = mul_mi<INV>(d);
        t3.x *= s3;
        t3.y *= s3;
        dst[0] = cadd(a[0], t1);
        dst[Ns] = cadd(t2, t3);
        dst[2 * Ns] = csub(t2, t3);
      } else {  // R == 5
        const T c1 = (T)0.30901699437494742410;   // cos(2 pi/5)
        const T c2 = (T)-0.80901699437494742410;  // cos(4 pi/5)
        const T s1 = (T)0.95105651629515357212;   // sin(2 pi/5)
        const T s2 = (T)0.58778525229247312917;   // sin(4 pi/5)
        C b1 = cadd(a[1], a[4]), b4 = csub(a[1], a[4]);
        C b2 = cadd(a[2], a[3]), b3 = csub(a[2], a[3]);
        C r1, r2;
        r1.x = a[0].x + c1 * b1.x + c2 * b2.x;
        r1.y = a[0].y + c1 * b1.y + c2 * b2.y;
        r2.x = a[0].x + c2 * b1.x + c1 * b2.x;
        r2.y = a[0].y + c2 * b1.y + c1 * b2.y;
        C i1, i2;  // (s1*b4 + s2*b3) and (s2*b4 - s1*b3), then times -i (fwd)
        i1.x = s1 * b4.x + s2 * b3.x;
        i1.y = s1 * b4.y + s2 * b3.y;
        i2.x = s2 * b4.x - s1 * b3.x;
        i2.y = s2 * b4.y - s1 * b3.y;
        i1 = mul_mi<INV>(i1);
        i2 = mul_mi<INV>(i2);
        C y0;
        y0.x = a[0].x + b1.x + b2.x;
        y0.y = a[0].y + b1.y + b2.y;
        dst[0] = y0;
        dst[Ns] = cadd(r1, i1);
        dst[4 * Ns] = csub(r1, i1);
        dst[2 * Ns] = cadd(r2, i2);
        dst[3 * Ns] = csub(r2, i2);
      }
    }
    __syncthreads();
    C *t = in;
    in = out;
    out = t;
    Ns *= R;
  }
  return in;
}

// ------------------------------------------------------------------------------------------
// Register-resident warp FFT for N = 32*N1 (N1 in {1,2,3,4,6,8,12,16,24,32}).
// Element n = lane + 32*m sits in lane `lane`, register m.  Step 1: an N1-point DFT over the
// lane's registers (compile-time Stockham passes of radix 4/2/3/5); step 2: twiddle register
// k1 by w_N^(lane*k1); step 3: a 32-point DFT across the lanes (5 decimation-in-frequency
// stages on xor shuffles).  Afterwards lane l, register k1 holds X[k1 + N1*bitrev5(l)].
// Twiddles come from the length-N table tw[m] = exp(-2 pi i m/N) (conjugated for INV).
// ------------------------------------------------------------------------------------------
struct RadixList {
  int n;
  int r[8];
};
__host__ __device__ constexpr RadixList radix_list(int N) {
  RadixList L{0, {0, 0, 0, 0, 0, 0, 0, 0}};
  int m = N;
  while (m % 4 == 0) { L.r[L.n++] = 4; m /= 4; }
  while (m % 2 == 0) { L.r[L.n++] = 2; m /= 2; }
  while (m % 3 == 0) { L.r[L.n++] = 3; m /= 3; }
  while (m % 5 == 0) { L.r[L.n++] = 5; m /= 5; }
  return L;
}

template <int R, bool INV, typename T>
__device__ __forceinline__ void dft_small(typename Cplx<T>::type (&a)[R]) {
  using C = typename Cplx<T>::type;
  if constexpr (R == 2) {
    C t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  } else if constexpr (R == 4) {
    C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    C t2 = cadd(a[1], a[3]), t3 = mul_mi<INV>(csub(a[1], a[3]));
    a[0] = cadd(t0, t2);
    a[1] = cadd(t1, t3);
    a[2] = csub(t0, t2);
    a[3] = csub(t1, t3);
  } else if constexpr (R == 3) {
    const T s3 = (T)0.86602540378443864676;
    C t1 = cadd(a[1], a[2]);
    C t2;
    t2.x = a[0].x - (T)0.5 * t1.x;
    t2.y = a[0].y - (T)0.5 * t1.y;
    C t3 = mul_mi<INV>(csub(a[1], a[2]));
    t3.x *= s3;
    t3.y *= s3;
    a[0] = cadd(a[0], t1);
    a[1] = cadd(t2, t3);
    a[2] = csub(t2, t3);
  } else if constexpr (R == 5) {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    C b1 = cadd(a[1], a[4]), b4 = csub(a[1], a[4]);
    C b2 = cadd(a[2], a[3]), b3 = csub(a[2], a[3]);
    C r1, r2, i1, i2, y0;
    r1.x = a[0].x + c1 * b1.x + c2 * b2.x;
    r1.y = a[0].y + c1 * b1.y + c2 * b2.y;
    r2.x = a[0].x + c2 * b1.x + c1 * b2.x;
    r2.y = a[0].y + c2 * b1.y + c1 * b2.y;
    i1.x = s1 * b4.x + s2 * b3.x;
    i1.y = s1 * b4.y + s2 * b3.y;
    i2.x = s2 * b4.x - s1 * b3.x;
    i2.y = s2 * b4.y - s1 * b3.y;
    i1 = mul_mi<INV>(i1);
    i2 = mul_mi<INV>(i2);
    y0.x = a[0].x + b1.x + b2.x;
    y0.y = a[0].y + b1.y + b2.y;
    a[0] = y0;
    a[1] = cadd(r1, i1);
    a[4] = csub(r1, i1);
    a[2] = cadd(r2, i2);
    a[3] = csub(r2, i2);
  }
}

template <bool INV, typename T>
__device__ __forceinline__ typename Cplx<T>::type twiddle(const typename Cplx<T>::type *__restrict__ tw,
                                                           int m) {
  typename Cplx<T>::type w = tw[m];
  if (INV) w.y = -w.y;
  return w;
}

// One Stockham pass of radix R over N1 registers (input x, output y); NS = product of earlier radices.
template <bool INV, typename T, int N1, int R, int NS>
__device__ __forceinline__ void reg_pass(const typename Cplx<T>::type (&x)[N1], typename Cplx<T>::type (&y)[N1],
                                         const typename Cplx<T>::type *__restrict__ tw) {
  using C = typename Cplx<T>::type;
  constexpr int NR = N1 / R;
#pragma unroll
  for (int jj = 0; jj < NR; ++jj) {
    const int k = jj % NS;
    C a[R];
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = x[jj + q * NR];
    if constexpr (NS > 1) {
#pragma unroll
      for (int q = 1; q < R; ++q) {
        // w_{NS*R}^(q*k) = w_N^(32 * q*k*N1/(NS*R)) for N = 32*N1
        if (k != 0) a[q] = cmul(a[q], twiddle<INV, T>(tw, 32 * q * k * (N1 / (NS * R))));
      }
    }
    dft_small<R, INV, T>(a);
#pragma unroll
    for (int q = 0; q < R; ++q) y[(jj / NS) * NS * R + k + q * NS] = a[q];
  }
}

template <bool INV, typename T, int N1, int P, int NS>
__device__ __forceinline__ void reg_fft_rec(typename Cplx<T>::type (&x)[N1],
                                            const typename Cplx<T>::type *__restrict__ tw) {
  using C = typename Cplx<T>::type;
  constexpr RadixList L = radix_list(N1);
  if constexpr (P < L.n) {
    constexpr int R = L.r[P];
    C y[N1];
    reg_pass<INV, T, N1, R, NS>(x, y, tw);
#pragma unroll
    for (int q = 0; q < N1; ++q) x[q] = y[q];
    reg_fft_rec<INV, T, N1, P + 1, NS * R>(x, tw);
  }
}

__device__ __forceinline__ int bitrev5(int l) { return (int)(__brev((unsigned)l) >> 27); }

template <bool INV, typename T, int N1>
__device__ __forceinline__ void warp_fft(typename Cplx<T>::type (&x)[N1], int lane,
                                         const typename Cplx<T>::type *__restrict__ tw) {
  using C = typename Cplx<T>::type;
  reg_fft_rec<INV, T, N1, 0, 1>(x, tw);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1)
    if (lane != 0) x[k1] = cmul(x[k1], twiddle<INV, T>(tw, lane * k1));
  C w5[5];
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    w5[s] = twiddle<INV, T>(tw, ((lane & (h - 1)) * (16 / h)) * N1);  // w_{2h}^(lane mod h)
  }
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const bool bottom = (lane & h) != 0;
#pragma unroll
    for (int q = 0; q < N1; ++q) {
      C o;
      o.x = __shfl_xor_sync(0xffffffffu, x[q].x, h);
      o.y = __shfl_xor_sync(0xffffffffu, x[q].y, h);
      x[q] = bottom ? cmul(csub(o, x[q]), w5[s]) : cadd(x[q], o);
    }
  }
}

// The lane-dependent twiddles of warp_fft for N = 32 N1 as a shared table [N1 + 4][32]: rows
// k1 - 1 = 0 .. N1 - 2 hold w_N^(lane k1), rows N1 - 1 .. N1 + 3 the five radix-2 stage factors,
// so a warp reads 32 consecutive entries (free of bank conflicts) instead of scattered global
// loads.  Filled by the whole block from the global table (the same values, so the same bits);
// the caller synchronises before use.
template <typename T, int N1>
__device__ __forceinline__ void fill_lane_twiddles(typename Cplx<T>::type *stw,
                                                   const typename Cplx<T>::type *__restrict__ tw) {
  for (int e = threadIdx.x; e < (N1 + 4) * 32; e += blockDim.x) {
    const int row = e >> 5, lane = e & 31;
    int m;
    if (row < N1 - 1) {
      m = lane * (row + 1);
    } else {
      const int h = 16 >> (row - (N1 - 1));
      m = ((lane & (h - 1)) * (16 / h)) * N1;
    }
    stw[e] = tw[m];
  }
}

// Bytes of that table, and whether a kernel of `bytes` dynamic shared memory a block keeps its
// blocks per SM (228 KB an SM, 1 KB reserved a block; at most 227 KB a block) with it added.
template <int N1, typename C = double2>
__host__ __device__ constexpr size_t lane_table_bytes() {
  return (size_t)(N1 + 4) * 32 * sizeof(C);
}
__host__ __device__ constexpr bool lane_table_fits(size_t bytes, size_t table) {
  return bytes + table <= 227 * 1024 && (228 * 1024) / (bytes + table + 1024) >= (228 * 1024) / (bytes + 1024);
}

// warp_fft with the lane-dependent twiddles read from a fill_lane_twiddles table.
template <bool INV, typename T, int N1>
__device__ __forceinline__ void warp_fft_lt(typename Cplx<T>::type (&x)[N1], int lane,
                                            const typename Cplx<T>::type *__restrict__ tw,
                                            const typename Cplx<T>::type *stw) {
  using C = typename Cplx<T>::type;
  reg_fft_rec<INV, T, N1, 0, 1>(x, tw);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1)
    if (lane != 0) x[k1] = cmul(x[k1], twiddle<INV, T>(stw, (k1 - 1) * 32 + lane));
  C w5[5];
#pragma unroll
  for (int s = 0; s < 5; ++s) w5[s] = twiddle<INV, T>(stw, (N1 - 1 + s) * 32 + lane);
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const bool bottom = (lane & h) != 0;
#pragma unroll
    for (int q = 0; q < N1; ++q) {
      C o;
      o.x = __shfl_xor_sync(0xffffffffu, x[q].x, h);
      o.y = __shfl_xor_sync(0xffffffffu, x[q].y, h);
      x[q] = bottom ? cmul(csub(o, x[q]), w5[s]) : cadd(x[q], o);
    }
  }
}

// ------------------------------------------------------------------------------------------
// Bounded device-side waits: every spin in this library counts iterations and gives up with
// an error flag instead of hanging (no trap, no unbounded loop).  A wait that gave up drains
// the copies still in flight with kDrainLimit polls before its block exits.
// ------------------------------------------------------------------------------------------
constexpr long long kSpinLimit = 1LL << 22;
constexpr long long kDrainLimit = 1LL << 28;

// Maximum that propagates NaN (fmax drops it): a NaN anywhere in a CFL or divergence
// reduction makes the result NaN, which the main-loop checks turn into an error code.
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }

// 1-D TMA bulk copies global -> shared, completed on an mbarrier (sm_90+ PTX, no tensor map,
// no multicast).  Source and destination must be 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bulk-group bookkeeping of the issuing thread (tensor stores shared -> global): commit the
// copies issued so far; wait until they have read their shared sources, or until complete.
// A shared source must be published to the async proxy first (fence_proxy_async_shared after
// the generic stores, then a barrier).
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Per-thread asynchronous copy of one BYTES-sized element (4, 8 or 16) global -> shared, with
// zero fill when `valid` is false (no byte is read then; src must still be a mapped address).
// Completed by cp_async_wait_all() in the issuing thread; a barrier publishes it to the block.
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void *dst, const void *src, bool valid) {
  static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async element size");
  const int n = valid ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(n)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES),
                 "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Wait for the given phase parity; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
  const uint32_t addr = smem_u32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace afid
