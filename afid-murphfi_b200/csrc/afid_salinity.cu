// afid_salinity.cu — the multi-resolution salinity scalar on the device (include/afid_salinity.h).
//
// Per substep (TimeMarcher.F90:50-63, 95, 138-144):
//   k_sal_step       ExplicitSalinity + ImplicitSalinity + SolveImpEqnUpdate_Sal fused per refined
//                    x-column (salinity.F90:268-453): one warp per column, RHS, CN solve, update
//   (K1 subtracts bycs * salc from the forcing along gAxis: AddSalBuoyancy, salinity.F90:494-506)
// after the projection:
//   k_sal_grad       dvx/dx, dvy/dy, dvz/dz at the coarse cell centres (InterpVelMgrd.F90:33-158)
//   k_sal_zint +     the three gradients interpolated to the refined cell centres
//   k_sal_to_ref     (interpolate_xyz_to_refined, HermiteInterpolations.F90:168-200); vxr is
//                    integrated along the column in the same block (InterpVelMgrd.F90:49-57)
//   k_sal_scan_y     first-guess plane at y = 0 (vy interpolated in x-z) + integration along y
//   k_sal_scan_z     first-guess plane at z = 0 (vz in x-y, when nzm > 1) + integration along z
//   k_sal_zc +       salc from the wall-extended refined salinity (InterpSalMultigrid,
//   k_sal_to_coarse  salinity.F90:455-492, per-target form of either coarse interpolation)
// Diagnostics: k_sal_cfl (CalcMaxCFL.F90:48-65), k_sal_prof_* (CalcSalStats, salinity.F90:508-667).
//
// Layout: refined fields are x-fastest like the coarse ones, (k, j, i) at k + ldr (j + nymr i),
// ldr = round_up(nxmr + 1, 8); vxr uses rows 0..nxmr (nxr faces), the others rows 0..nxmr-1.
// Every stencil is a per-target table (first source row + 4 weights); along x the sources are
// wall-extended columns whose ghost rows are formed on the fly.
#include <cuda_runtime.h>

#include "afid_device.cuh"
#include "afid_internal.h"
#include "afid_k1.cuh"

namespace afid {

namespace {

__device__ __forceinline__ int wrapmod(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// Wall-extended coarse column (InterpVelMgrd.F90:40-41, 75-76, 107-108): row -1 is
// (1 - 2 inslwS) row 0, row nxm is (1 - 2 inslwN) row nxm-1, rows -2 and nxm+1 are zero.
__device__ __forceinline__ double coarse_ext(const double *__restrict__ col, int r, int nxm, double fs, double fn) {
  if (r >= 0 && r < nxm) return __ldg(col + r);
  if (r == -1) return fs * __ldg(col);
  if (r == nxm) return fn * __ldg(col + nxm - 1);
  return 0.0;
}

// Wall-extended refined salinity (salinity.F90:462-481): row -1 is 2 salbp - sal(0) with SfixS
// (else sal(0)), row nxmr is 2 saltp - sal(nxmr-1) with SfixN (else sal(nxmr-1)); -2 and nxmr+1
// are zero.
// The plate values are read only for the ghost rows.
__device__ __forceinline__ double sal_ext(const double *__restrict__ col, int r, int n, int sfixs, int sfixn,
                                          const double *__restrict__ bp, const double *__restrict__ tp) {
  if (r >= 0 && r < n) return __ldg(col + r);
  if (r == -1) return sfixs ? 2.0 * __ldg(bp) - __ldg(col) : __ldg(col);
  if (r == n) return sfixn ? 2.0 * __ldg(tp) - __ldg(col + n - 1) : __ldg(col + n - 1);
  return 0.0;
}

// ------------------------------------------------------------------------------------------
// k_sal_grad: one thread per coarse cell (k < nxm) of the padded field.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_sal_grad(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
               const double *__restrict__ vz, double *__restrict__ gx, double *__restrict__ gy,
               double *__restrict__ gz) {
  const size_t n = (size_t)g.ldx * g.nym * g.nzm;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % g.ldx);
    if (k >= g.nxm) continue;
    const size_t col = e / g.ldx;
    const int j = (int)(col % g.nym), i = (int)(col / g.nym);
    const size_t ojp = col_off(g, wrap_inc(j, g.nym), i) + k, oip = col_off(g, j, wrap_inc(i, g.nzm)) + k;
    gx[e] = (vx[e + 1] - vx[e]) * __ldg(t.udx3m + k);  // InterpVelMgrd.F90:37
    gy[e] = (vy[ojp] - vy[e]) * g.dy;                   // :72
    gz[e] = (vz[oip] - vz[e]) * g.dz;                   // :156
  }
}

// ------------------------------------------------------------------------------------------
// Coarse -> refined interpolation of the three velocity gradients in two passes, contracting z,
// then y, then x exactly as qv2 / qv1 of HermiteInterpolations.F90:186-196:
//   k_sal_zint   T_f(r, jc, ir) = sum_c wz_c(ir) g_f(r, jc, sz(ir) + c), block per column;
//   k_sal_to_ref warp per refined column (jr, ir): q_f(r) = sum_b wy_b(jr) T_f(r, sy(jr) + b, ir)
//                gives a wall-extended coarse column per gradient in shared memory, the x
//                contraction yields the refined gradients, and dvx/dx is integrated along the
//                column (vxr(1) = 0, InterpVelMgrd.F90:48-57); dvy/dy and dvz/dz go to scratch
//                for the y and z integrations.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_sal_zint(Geom g, SalGeom sg, SalTables st, const double *__restrict__ gx, const double *__restrict__ gy,
               const double *__restrict__ gz, double *__restrict__ tz) {
  // block per output column (jc, ir): the four source columns and weights are block constants
  const int jc = blockIdx.x % g.nym, ir = blockIdx.x / g.nym;
  const size_t n = (size_t)g.ldx * g.nym * sg.nzmr;
  const size_t out = ((size_t)jc + (size_t)g.nym * ir) * g.ldx;
  const int sz = __ldg(st.st[2] + ir);
  double w[4];
  size_t o[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    w[c] = __ldg(st.w[2] + 4 * ir + c);
    o[c] = ((size_t)jc + (size_t)g.nym * wrapmod(sz + c, g.nzm)) * g.ldx;
  }
  const double *src[3] = {gx, gy, gz};
  for (int r = threadIdx.x; r < g.nxm; r += blockDim.x) {
#pragma unroll
    for (int f = 0; f < 3; ++f)
      tz[(size_t)f * n + out + r] = __ldg(src[f] + o[0] + r) * w[0] + __ldg(src[f] + o[1] + r) * w[1] +
                                    __ldg(src[f] + o[2] + r) * w[2] + __ldg(src[f] + o[3] + r) * w[3];
  }
}

// Warp per refined column, four columns per block, no block barriers: the y contraction of the
// four T columns goes to the warp's shared rows, then 32-row strips are contracted in x and dvx/dx
// is integrated by a warp scan whose total carries to the next strip.
constexpr int kToRefWarps = 4;

__global__ void __launch_bounds__(32 * kToRefWarps)
    k_sal_to_ref(Geom g, SalGeom sg, SalTables st, const double *__restrict__ tz, double *__restrict__ vxr,
                 double *__restrict__ gyr, double *__restrict__ gzr) {
  extern __shared__ __align__(16) double sm_to_ref[];
  const int nxm = g.nxm, L = nxm + 4;  // extended rows -2 .. nxm+1 at 0 .. nxm+3
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * kToRefWarps + warp;
  if (col >= sg.nymr * sg.nzmr) return;  // whole warps only: nothing below synchronises the block
  double *qx = sm_to_ref + (size_t)warp * 3 * L, *qy = qx + L, *qz = qy + L;
  const int jr = col % sg.nymr, ir = col / sg.nymr;
  const int sy = __ldg(st.st[1] + jr);
  const size_t n = (size_t)g.ldx * g.nym * sg.nzmr;
  double wy[4];
  size_t co[4];  // T columns (sy + b, ir)
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    wy[b] = __ldg(st.w[1] + 4 * jr + b);
    co[b] = ((size_t)wrapmod(sy + b, g.nym) + (size_t)g.nym * ir) * g.ldx;
  }
  for (int r = lane; r < nxm; r += 32) {
    double q[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const double *t = tz + (size_t)f * n + r;
      q[f] = __ldg(t + co[0]) * wy[0] + __ldg(t + co[1]) * wy[1] + __ldg(t + co[2]) * wy[2] + __ldg(t + co[3]) * wy[3];
    }
    qx[r + 2] = q[0];
    qy[r + 2] = q[1];
    qz[r + 2] = q[2];
  }
  __syncwarp();
  if (lane < 3) {
    // ghost rows: the wall rule (a factor +-1) commutes exactly with the y-z contraction
    double *q = lane == 0 ? qx : (lane == 1 ? qy : qz);
    q[0] = 0.0;
    q[1] = (double)(1 - 2 * g.inslws) * q[2];
    q[nxm + 2] = (double)(1 - 2 * g.inslwn) * q[nxm + 1];
    q[nxm + 3] = 0.0;
  }
  __syncwarp();
  const size_t roff = ((size_t)jr + (size_t)sg.nymr * ir) * sg.ldr;
  const int nxmr = sg.nxmr;
  double carry = 0.0;
  if (lane == 0) vxr[roff] = 0.0;  // InterpVelMgrd.F90:48
  for (int k0 = 0; k0 < nxmr; k0 += 32) {
    const int kr = k0 + lane;
    double d = 0.0;
    if (kr < nxmr) {
      const int p = __ldg(st.st[0] + kr) + 2;
      const double2 w01 = __ldg(reinterpret_cast<const double2 *>(st.w[0] + 4 * kr));
      const double2 w23 = __ldg(reinterpret_cast<const double2 *>(st.w[0] + 4 * kr + 2));
      const double vxg = qx[p] * w01.x + qx[p + 1] * w01.y + qx[p + 2] * w23.x + qx[p + 3] * w23.y;
      gyr[roff + kr] = qy[p] * w01.x + qy[p + 1] * w01.y + qy[p + 2] * w23.x + qy[p + 3] * w23.y;
      gzr[roff + kr] = qz[p] * w01.x + qz[p + 1] * w01.y + qz[p + 2] * w23.x + qz[p + 3] * w23.y;
      d = vxg * __ldg(st.lxa + kr);  // InterpVelMgrd.F90:53-54
    }
    // vxr(kr+1) = vxr(kr) + d(kr): inclusive scan of the strip plus the carried total
    double incl = d;
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, incl, h);
      if (lane >= h) incl += o;
    }
    if (kr < nxmr) vxr[roff + kr + 1] = carry + incl;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
}

// ------------------------------------------------------------------------------------------
// k_sal_scan_y: thread per (kr, ir).  vyr at the plane y = 0 (jcr0 = 1) is vy(:, 1, :)
// interpolated in x-z (InterpVelMgrd.F90:99-116: z contracted first, then x); then
// vyr(jr+1) = vyr(jr) + dvy/dy(jr) / dyr (:124-131).  One rank: the MPI_SCAN correction is zero.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_sal_scan_y(Geom g, SalGeom sg, SalTables st, const double *__restrict__ vy, const double *__restrict__ gyr,
                 double *__restrict__ vyr) {
  const int kr = blockIdx.x * blockDim.x + threadIdx.x, ir = blockIdx.y;
  if (kr >= sg.nxmr) return;
  const int sx = __ldg(st.st[0] + kr), sz = __ldg(st.st[2] + ir);
  const double fs = (double)(1 - 2 * g.inslws), fn = (double)(1 - 2 * g.inslwn);
  double v = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    double q1 = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double *col = vy + col_off(g, 0, wrapmod(sz + c, g.nzm));
      const double e = coarse_ext(col, sx + a, g.nxm, fs, fn) * __ldg(st.w[2] + 4 * ir + c);
      q1 = (c == 0) ? e : q1 + e;
    }
    const double e = q1 * __ldg(st.w[0] + 4 * kr + a);
    v = (a == 0) ? e : v + e;
  }
  size_t o = (size_t)sg.nymr * ir * sg.ldr + kr;
  vyr[o] = v;
  for (int jr = 0; jr + 1 < sg.nymr; ++jr) {
    v = v + __ldg(gyr + o) * sg.lya;
    o += sg.ldr;
    vyr[o] = v;
  }
}

// ------------------------------------------------------------------------------------------
// k_sal_scan_z: thread per (kr, jr).  vzr at the plane z = 0 (icr0 = 1) is vz(:, :, 1)
// interpolated in x-y (InterpVelMgrd.F90:181-198: y first, then x), only when nzm > 1 (the
// reference's `ic0 < xend(3)`); then vzr(ir+1) = vzr(ir) + dvz/dz(ir) / dzr (:206-213).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_sal_scan_z(Geom g, SalGeom sg, SalTables st, const double *__restrict__ vz, const double *__restrict__ gzr,
                 double *__restrict__ vzr) {
  const int kr = blockIdx.x * blockDim.x + threadIdx.x, jr = blockIdx.y;
  if (kr >= sg.nxmr) return;
  double v = 0.0;
  if (g.nzm > 1) {
    const int sx = __ldg(st.st[0] + kr), sy = __ldg(st.st[1] + jr);
    const double fs = (double)(1 - 2 * g.inslws), fn = (double)(1 - 2 * g.inslwn);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      double q1 = 0.0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const double *col = vz + col_off(g, wrapmod(sy + b, g.nym), 0);
        const double e = coarse_ext(col, sx + a, g.nxm, fs, fn) * __ldg(st.w[1] + 4 * jr + b);
        q1 = (b == 0) ? e : q1 + e;
      }
      const double e = q1 * __ldg(st.w[0] + 4 * kr + a);
      v = (a == 0) ? e : v + e;
    }
  }
  const size_t plane = (size_t)sg.nymr * sg.ldr;
  size_t o = (size_t)jr * sg.ldr + kr;
  vzr[o] = v;
  for (int ir = 0; ir + 1 < sg.nzmr; ++ir) {
    v = v + __ldg(gzr + o) * sg.lza;
    o += plane;
    vzr[o] = v;
  }
}

// ------------------------------------------------------------------------------------------
// Refined -> coarse interpolation of salinity (InterpSalMultigrid) in two passes, z, then y,
// then x as HermiteInterpolations.F90:270-284:
//   k_sal_zc         U(rr, jr, ic) = sum_c wz_c(ic) S_ext(rr, jr, sz(ic) + c) for the extended
//                    refined rows rr = -2 .. nxmr+1 (stored at rr + 2, stride ldu), block per
//                    column; the plate ghosts are formed per refined column as the reference
//                    does before its contraction (salinity.F90:462-481);
//   k_sal_to_coarse  warp per coarse column (j, i): U2(rr) = sum_b wy_b(j) U(rr, sy(j) + b, i)
//                    in shared memory, then salc(k) = sum_a wx_a(k) U2(sx(k) + a).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_sal_zc(Geom g, SalGeom sg, SalTables st, const double *__restrict__ sal, double *__restrict__ u) {
  // block per output column (jr, ic): the four refined source columns, their plates and the
  // weights are block constants
  const int jr = blockIdx.x % sg.nymr, ic = blockIdx.x / sg.nymr;
  const int sz = __ldg(st.st[5] + ic);
  double w[4];
  const double *colp[4];
  size_t pl[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    w[c] = __ldg(st.w[5] + 4 * ic + c);
    pl[c] = (size_t)jr + (size_t)sg.nymr * wrapmod(sz + c, sg.nzmr);
    colp[c] = sal + pl[c] * sg.ldr;
  }
  double *out = u + ((size_t)jr + (size_t)sg.nymr * ic) * sg.ldu;
  for (int q = threadIdx.x; q < sg.nxmr + 4; q += blockDim.x) {
    const int rr = q - 2;
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double s = sal_ext(colp[c], rr, sg.nxmr, sg.sfixs, sg.sfixn, st.salbp + pl[c], st.saltp + pl[c]) * w[c];
      v = (c == 0) ? s : v + s;
    }
    out[q] = v;
  }
}

constexpr int kToCoarseWarps = 4;

__global__ void __launch_bounds__(32 * kToCoarseWarps)
    k_sal_to_coarse(Geom g, SalGeom sg, SalTables st, const double *__restrict__ u, double *__restrict__ salc) {
  // warp per coarse column (j, i), four per block, no block barriers
  extern __shared__ __align__(16) double sm_to_c[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = blockIdx.x * kToCoarseWarps + warp;
  if (col >= g.nym * g.nzm) return;
  const int nrows = sg.nxmr + 4;
  double *q = sm_to_c + (size_t)warp * nrows;
  const int j = col % g.nym, i = col / g.nym;
  const int sy = __ldg(st.st[4] + j);
  double wy[4];
  size_t co[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    wy[b] = __ldg(st.w[4] + 4 * j + b);
    co[b] = ((size_t)wrapmod(sy + b, sg.nymr) + (size_t)sg.nymr * i) * sg.ldu;
  }
  for (int r = lane; r < nrows; r += 32)
    q[r] = __ldg(u + co[0] + r) * wy[0] + __ldg(u + co[1] + r) * wy[1] + __ldg(u + co[2] + r) * wy[2] +
           __ldg(u + co[3] + r) * wy[3];
  __syncwarp();
  const size_t c0 = col_off(g, j, i);
  for (int k = lane; k < g.nxm; k += 32) {
    const int p = __ldg(st.st[3] + k) + 2;
    const double2 w01 = __ldg(reinterpret_cast<const double2 *>(st.w[3] + 4 * k));
    const double2 w23 = __ldg(reinterpret_cast<const double2 *>(st.w[3] + 4 * k + 2));
    salc[c0 + k] = q[p] * w01.x + q[p + 1] * w01.y + q[p + 2] * w23.x + q[p + 3] * w23.y;
  }
}

// ------------------------------------------------------------------------------------------
// k_sal_step: one warp per refined column (j, i), four columns per block, no block barriers.
// Lane l owns rows l, l + 32, ...: it forms the explicit terms and the RHS of its rows
// (ExplicitSalinity, salinity.F90:309-364; ImplicitAndUpdate :375-402) from coalesced loads of
// the column and its neighbours (only the column itself is read at k +- 1), updates rusal in
// place and puts the RHS, scaled by 1/(1 - ac betadx), into the warp's chunk-layout rows in
// shared memory; the warp then solves the CN system with the factor tables of k_cn_tables
// (SolveImpEqnUpdate_Sal :408-452) and writes sal_o = sal + increment.  In 2-D the z neighbours
// are the column itself and those terms vanish; they are left out.
// ------------------------------------------------------------------------------------------
constexpr int kSalStepWarps = 4;

__host__ __device__ inline size_t sal_step_smem(int MR, bool two_d) {
  (void)two_d;
  return (size_t)kSalStepWarps * chunk_ld(MR) * MR * sizeof(double);
}

template <int MR, bool TWO_D>
__global__ void __launch_bounds__(32 * kSalStepWarps)
    k_sal_step(SalGeom sg, SalTables st, const StepCoef *__restrict__ sc_all, int ns, const double *__restrict__ cn_tab,
               const double *__restrict__ sal, const double *__restrict__ vxr, const double *__restrict__ vyr,
               const double *__restrict__ vzr, double *__restrict__ rusal, double *__restrict__ sal_o) {
  constexpr int LD = chunk_ld(MR);
  constexpr int B = MR < 2 ? MR : 2;  // rows per lane whose operands are loaded together
  static_assert(MR % B == 0, "row batches must tile the column");
  extern __shared__ __align__(16) double smem_sal[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nymr = sg.nymr, nzmr = sg.nzmr, n = sg.nxmr;
  const int col = blockIdx.x * kSalStepWarps + warp;
  if (col >= nymr * nzmr) return;  // whole warps only: nothing below synchronises the block
  double *s_rhs = smem_sal + (size_t)warp * LD * MR;
  const int j = col % nymr, i = col / nymr;
  auto off = [&](int jj, int ii) { return ((size_t)jj + (size_t)nymr * ii) * sg.ldr; };
  const size_t c0 = off(j, i), ojp = off(wrap_inc(j, nymr), i), ojm = off(wrap_dec(j, nymr), i);
  const size_t oip = off(j, wrap_inc(i, nzmr)), oim = off(j, wrap_dec(i, nzmr));
  const StepCoef sc = sc_all[ns];
  const double *T = cn_tab + (size_t)ns * cn_table_size(MR);
  const double bp = __ldg(st.salbp + col), tp = __ldg(st.saltp + col);
  const double alpec = sc.alpec;  // al / pecs (salinity.F90:374)
  // operands of one row: sal(k), sal(k-1), sal(k+1), sal(j+-1), vxr(k), vxr(k+1), vyr(j), vyr(j+1),
  // rusal, then (3-D) sal(i+-1), vzr(i), vzr(i+1)
  constexpr int NV = TWO_D ? 9 : 13;
#pragma unroll 1
  for (int p0 = 0; p0 < MR; p0 += B) {
    double v[B][NV];
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int k = lane + 32 * (p0 + q);
      const int kk = k < n ? k : n - 1;  // rows past the column read a valid row and are discarded
      v[q][0] = __ldg(sal + c0 + kk);
      v[q][1] = kk > 0 ? __ldg(sal + c0 + kk - 1) : 0.0;
      v[q][2] = kk < n - 1 ? __ldg(sal + c0 + kk + 1) : 0.0;
      v[q][3] = __ldg(sal + ojp + kk);
      v[q][4] = __ldg(sal + ojm + kk);
      v[q][5] = __ldg(vxr + c0 + kk);
      v[q][6] = __ldg(vxr + c0 + kk + 1);
      v[q][7] = __ldg(vyr + c0 + kk);
      v[q][8] = __ldg(vyr + ojp + kk);
      if constexpr (!TWO_D) {
        v[q][9] = __ldg(sal + oip + kk);
        v[q][10] = __ldg(sal + oim + kk);
        v[q][11] = __ldg(vzr + c0 + kk);
        v[q][12] = __ldg(vzr + oip + kk);
      }
    }
    double ru[B];
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int k = lane + 32 * (p0 + q);
      ru[q] = rusal[c0 + (k < n ? k : n - 1)];
    }
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int k = lane + 32 * (p0 + q);
      double rhs_s = 0.0;  // identity rows k >= n
      if (k < n) {
        const double sc_ = v[q][0], sm = v[q][1], sp = v[q][2], sjp = v[q][3], sjm = v[q][4];
        const double vx0 = v[q][5], vx1 = v[q][6], vy0 = v[q][7], vy1 = v[q][8];
        const double ux = __ldg(st.udx3mr + k);
        double hsx;
        if (k == 0)
          hsx = (vx1 * (sp + sc_) - vx0 * 2.0 * bp) * ux * 0.5;
        else if (k == n - 1)
          hsx = (vx1 * 2.0 * tp - vx0 * (sc_ + sm)) * ux * 0.5;
        else
          hsx = (vx1 * (sp + sc_) - vx0 * (sc_ + sm)) * ux * 0.5;
        const double hsy = (vy1 * (sjp + sc_) - vy0 * (sc_ + sjm)) * sg.udyr;
        const double dyys = (sjp - 2.0 * sc_ + sjm) * sg.udyrq;
        double hsal;
        if constexpr (TWO_D) {
          hsal = -(hsx + hsy) + dyys;
        } else {
          const double sip = v[q][9], sim = v[q][10], vz0 = v[q][11], vz1 = v[q][12];
          const double hsz = (vz1 * (sip + sc_) - vz0 * (sc_ + sim)) * sg.udzr;
          const double dzzs = (sip - 2.0 * sc_ + sim) * sg.udzrq;
          hsal = -(hsx + hsy + hsz) + dyys + dzzs;
        }
        const double a_p = __ldg(st.ap + k), a_c = __ldg(st.ac + k), a_m = __ldg(st.am + k);
        double dxxs;
        if (k == 0)
          dxxs = sp * a_p + sc_ * a_c - (a_p + a_c) * bp * sg.sfixs;
        else if (k == n - 1)
          dxxs = sc_ * a_c + sm * a_m - (a_m + a_c) * tp * sg.sfixn;
        else
          dxxs = sp * a_p + sc_ * a_c + sm * a_m;
        const double rhs = (sc.ga * hsal + sc.ro * ru[q] + alpec * dxxs) * sc.dt;
        rusal[c0 + k] = hsal;
        rhs_s = rhs * __ldg(T + k);
      }
      s_rhs[(k % MR) * LD + k / MR] = rhs_s;
    }
  }
  __syncwarp();
  cn_solve_chunk<MR, LD>(s_rhs, T, lane);
  __syncwarp();
#pragma unroll 4
  for (int p = 0; p < MR; ++p) {
    const int k = lane + 32 * p;
    if (k < n) sal_o[c0 + k] = __ldg(sal + c0 + k) + s_rhs[(k % MR) * LD + k / MR];  // column re-read hits L1/L2
  }
}

template <int MR>
cudaError_t launch_sal_step_M(const SalCtx &S, cudaStream_t stream, int ns) {
  const bool two_d = S.sg.nzmr == 1;
  const size_t smem = sal_step_smem(MR, two_d);
  const int ncol = S.sg.nymr * S.sg.nzmr;
  const int nblk = (ncol + kSalStepWarps - 1) / kSalStepWarps;
  if (two_d)
    k_sal_step<MR, true><<<nblk, 32 * kSalStepWarps, smem, stream>>>(S.sg, S.st, S.sc, ns, S.cn_tab, S.sal, S.vxr,
                                                                     S.vyr, S.vzr, S.rusal, S.sal_o);
  else
    k_sal_step<MR, false><<<nblk, 32 * kSalStepWarps, smem, stream>>>(S.sg, S.st, S.sc, ns, S.cn_tab, S.sal, S.vxr,
                                                                      S.vyr, S.vzr, S.rusal, S.sal_o);
  return cudaGetLastError();
}

//                    salinity.F90:455-492, per-target form of either coarse interpolation)
// ------------------------------------------------------------------------------------------
// Diagnostics
// ------------------------------------------------------------------------------------------
// CalcMaxCFL.F90:48-65: max over refined cells of |vz|/dz + |vy|/dy + |vx|/dx at the centre.
// Non-negative doubles order like their bit patterns, so the maximum is an integer atomicMax.
__global__ void __launch_bounds__(256)
    k_sal_cfl(SalGeom sg, SalTables st, const double *__restrict__ vxr, const double *__restrict__ vyr,
              const double *__restrict__ vzr, unsigned long long *__restrict__ out) {
  // blocks walk whole refined columns; a thread per row
  const int ncol = sg.nymr * sg.nzmr;
  double m = 0.0;
  for (int col = blockIdx.x; col < ncol; col += gridDim.x) {
    const int j = col % sg.nymr, i = col / sg.nymr;
    const size_t o = (size_t)col * sg.ldr;
    const size_t ojp = ((size_t)wrap_inc(j, sg.nymr) + (size_t)sg.nymr * i) * sg.ldr;
    const size_t oip = ((size_t)j + (size_t)sg.nymr * wrap_inc(i, sg.nzmr)) * sg.ldr;
    for (int k = threadIdx.x; k < sg.nxmr; k += blockDim.x) {
      const double q = fabs((__ldg(vzr + o + k) + __ldg(vzr + oip + k)) * 0.5 * sg.dzr) +
                       fabs((__ldg(vyr + o + k) + __ldg(vyr + ojp + k)) * 0.5 * sg.dyr) +
                       fabs((__ldg(vxr + o + k) + __ldg(vxr + o + k + 1)) * 0.5 * __ldg(st.udx3mr + k));
      m = nan_max(m, q);
    }
  }
#pragma unroll
  for (int h = 16; h > 0; h >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, h));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = nan_max(m, wm[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

// CalcSalStats / CalcDissipationSal (salinity.F90:537-566, 621-655): block b sums columns
// b, b + nb, ... for every row k; partial[(b * 6 + q) * nxmr + k].
__global__ void __launch_bounds__(256)
    k_sal_prof_partial(SalGeom sg, SalTables st, const double *__restrict__ sal, const double *__restrict__ vxr,
                       const double *__restrict__ vyr, const double *__restrict__ vzr, double *__restrict__ partial) {
  const int n = sg.nxmr, ncol = sg.nymr * sg.nzmr;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double a[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double tdx = __ldg(st.tdxr + k);
    for (int col = blockIdx.x; col < ncol; col += gridDim.x) {
      const int j = col % sg.nymr, i = col / sg.nymr;
      const size_t o = (size_t)col * sg.ldr;
      const size_t ojp = ((size_t)wrap_inc(j, sg.nymr) + (size_t)sg.nymr * i) * sg.ldr;
      const size_t ojm = ((size_t)wrap_dec(j, sg.nymr) + (size_t)sg.nymr * i) * sg.ldr;
      const size_t oip = ((size_t)j + (size_t)sg.nymr * wrap_inc(i, sg.nzmr)) * sg.ldr;
      const size_t oim = ((size_t)j + (size_t)sg.nymr * wrap_dec(i, sg.nzmr)) * sg.ldr;
      const double s = sal[o + k];
      a[0] += s;
      a[1] += s * s;
      a[2] += 0.5 * (vxr[o + k] + vxr[o + k + 1]) * s;
      a[3] += 0.5 * (vyr[o + k] + vyr[ojp + k]) * s;
      a[4] += 0.5 * (vzr[o + k] + vzr[oip + k]) * s;
      const double dz_ = (sal[oip + k] - sal[oim + k]) * 0.5 * sg.dzr;
      const double dy_ = (sal[ojp + k] - sal[ojm + k]) * 0.5 * sg.dyr;
      double dx_;
      if (k == 0) {
        const double bp = __ldg(st.salbp + col);
        dx_ = (sal[o + 1] - s + 2.0 * sg.sfixs * (s - bp)) * tdx;
      } else if (k == n - 1) {
        const double tp = __ldg(st.saltp + col);
        dx_ = (s - sal[o + k - 1] + 2.0 * sg.sfixn * (tp - s)) * tdx;
      } else {
        dx_ = (sal[o + k + 1] - sal[o + k - 1]) * tdx;
      }
      a[5] += dz_ * dz_;
      a[5] += dy_ * dy_;
      a[5] += dx_ * dx_;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) partial[((size_t)blockIdx.x * 6 + q) * n + k] = a[q];
  }
}

// Sum the block partials in block order and turn sums into averages (salinity.F90:578-587).
__global__ void k_sal_prof_reduce(SalGeom sg, const double *__restrict__ partial, int nb, double *__restrict__ out) {
  const int n = sg.nxmr;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 6 * n) return;
  const int q = e / n, k = e % n;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += partial[((size_t)b * 6 + q) * n + k];
  const double inyz = 1.0 / sg.nymr / sg.nzmr;
  if (q == 1)
    s = sqrt(s * inyz);
  else if (q == 5)
    s = s / sg.pecs * inyz;
  else
    s = s * inyz;
  out[e] = s;
}

int grid_for(size_t n, int tpb) {
  const size_t b = (n + tpb - 1) / tpb;
  return (int)(b < (size_t)148 * 16 ? b : (size_t)148 * 16);
}

}  // namespace

int sal_prof_blocks(const SalGeom &sg) {
  const int ncol = sg.nymr * sg.nzmr;
  return ncol < 148 * 4 ? ncol : 148 * 4;
}

cudaError_t launch_sal_step(const LaunchCtx &L, const SalCtx &S, int ns) {
  switch (S.sg.MR) {
    case 1: return launch_sal_step_M<1>(S, L.stream, ns);
    case 2: return launch_sal_step_M<2>(S, L.stream, ns);
    case 4: return launch_sal_step_M<4>(S, L.stream, ns);
    case 8: return launch_sal_step_M<8>(S, L.stream, ns);
    case 12: return launch_sal_step_M<12>(S, L.stream, ns);
    case 16: return launch_sal_step_M<16>(S, L.stream, ns);
    case 24: return launch_sal_step_M<24>(S, L.stream, ns);
    case 32: return launch_sal_step_M<32>(S, L.stream, ns);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sal_interp(const LaunchCtx &L, const SalCtx &S, const double *vx, const double *vy,
                              const double *vz) {
  const Geom &g = L.g;
  const size_t nc = (size_t)g.ldx * g.nym * g.nzm;
  k_sal_grad<<<grid_for(nc, 256), 256, 0, L.stream>>>(g, L.t, vx, vy, vz, S.gx, S.gy, S.gz);
  k_sal_zint<<<g.nym * S.sg.nzmr, 128, 0, L.stream>>>(g, S.sg, S.st, S.gx, S.gy, S.gz, S.tmp);
  const size_t smem = (size_t)kToRefWarps * 3 * (g.nxm + 4) * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_sal_to_ref, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int ncr = S.sg.nymr * S.sg.nzmr;
  k_sal_to_ref<<<(ncr + kToRefWarps - 1) / kToRefWarps, 32 * kToRefWarps, smem, L.stream>>>(g, S.sg, S.st, S.tmp,
                                                                                            S.vxr, S.gyr, S.gzr);
  const dim3 gy((S.sg.nxmr + 127) / 128, S.sg.nzmr), gz((S.sg.nxmr + 127) / 128, S.sg.nymr);
  k_sal_scan_y<<<gy, 128, 0, L.stream>>>(g, S.sg, S.st, vy, S.gyr, S.vyr);
  k_sal_scan_z<<<gz, 128, 0, L.stream>>>(g, S.sg, S.st, vz, S.gzr, S.vzr);
  k_sal_zc<<<S.sg.nymr * g.nzm, 128, 0, L.stream>>>(g, S.sg, S.st, S.sal, S.tmp);
  const size_t smc = (size_t)kToCoarseWarps * (S.sg.nxmr + 4) * sizeof(double);
  const int ncc = g.nym * g.nzm;
  k_sal_to_coarse<<<(ncc + kToCoarseWarps - 1) / kToCoarseWarps, 32 * kToCoarseWarps, smc, L.stream>>>(
      g, S.sg, S.st, S.tmp, S.salc);
  return cudaGetLastError();
}

cudaError_t launch_sal_cfl(const LaunchCtx &L, const SalCtx &S) {
  cudaError_t e = cudaMemsetAsync(S.red, 0, sizeof(unsigned long long), L.stream);
  if (e != cudaSuccess) return e;
  const int ncol = S.sg.nymr * S.sg.nzmr;
  k_sal_cfl<<<ncol < 148 * 8 ? ncol : 148 * 8, 256, 0, L.stream>>>(S.sg, S.st, S.vxr, S.vyr, S.vzr, S.red);
  return cudaGetLastError();
}

cudaError_t launch_sal_profiles(const LaunchCtx &L, const SalCtx &S, double *out) {
  const int nb = sal_prof_blocks(S.sg);
  k_sal_prof_partial<<<nb, 256, 0, L.stream>>>(S.sg, S.st, S.sal, S.vxr, S.vyr, S.vzr, S.partial);
  const int ne = 6 * S.sg.nxmr;
  k_sal_prof_reduce<<<(ne + 255) / 256, 256, 0, L.stream>>>(S.sg, S.partial, nb, out);
  return cudaGetLastError();
}

size_t sal_step_smem_bytes(int MR, bool two_d) { return sal_step_smem(MR, two_d); }

}  // namespace afid
