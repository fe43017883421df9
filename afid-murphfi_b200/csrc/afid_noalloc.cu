// afid_noalloc.cu — volume statistics (Nusselt number, kinetic energy, mean temperature) for
// callers that cannot allocate device memory.
//
// Who needs this: code that owns the GPU's memory itself — a Fortran main program with its own
// device pool, a host application running under a custom or capped allocator, or a monitor
// injected into someone else's run — cannot let a library call cudaMalloc behind its back,
// and may not even be allowed to (the allocation would bypass its accounting or fail under
// its cap).  afid_gpu_globals needs a per-context device buffer for its partial sums; this
// entry point computes the same quantities on device fields the caller already owns and
// keeps its partial sums in a fixed static array that is part of the loaded library.
//
// The scratch array below is a file-scope __device__ array: every GPU that loads the library
// holds AFID_NOALLOC_SCRATCH_BYTES of it until the process exits.  All calls share it, it
// keeps the last call's contents, and two calls that overlap on the GPU (different streams or
// threads without ordering) race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "afid_gpu.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[AFID_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};  // device address of g_noalloc_scratch, per device
void *g_scratch_ctx[kMaxDevices] = {};   // the context each address was looked up in

// One warp per (j,i) column: the three g3rc-weighted sums of GlobalQuantities.F90:39-60 for
// that column go to partial[3*col + q], so every partial is rewritten on every call.
__global__ void __launch_bounds__(256)
    k_noalloc_column_sums(int nxm, int nym, int nzm, int ldx, const double *__restrict__ vx,
                          const double *__restrict__ vy, const double *__restrict__ vz,
                          const double *__restrict__ temp, const double *__restrict__ g3rc,
                          double *__restrict__ partial) {
  const int lane = threadIdx.x & 31;
  const long long col = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= (long long)nym * nzm) return;
  const size_t c = (size_t)col * ldx;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int k = lane; k < nxm; k += 32) {
    const double fac2 = g3rc[k];
    const double vxcen = (vx[c + k] + vx[c + k + 1]) * 0.5;
    const double tc = temp[c + k];
    s0 += tc * vxcen * fac2;
    s1 += fac2 * (vz[c + k] * vz[c + k] + vy[c + k] * vy[c + k] + vx[c + k] * vx[c + k]);
    s2 += tc * fac2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    partial[3 * col + 0] = s0;
    partial[3 * col + 1] = s1;
    partial[3 * col + 2] = s2;
  }
}

// Single block: sums the column partials in a fixed order and writes
// out3 = {1 + sqrt(ra_pr) * vol * sum0, 0.5 * vol * sum1, vol * sum2} (GlobalQuantities.F90:79, 87-91).
__global__ void __launch_bounds__(256)
    k_noalloc_finish(const double *__restrict__ partial, long long ncol, double vol, double sqrt_ra_pr,
                     double *__restrict__ out3) {
  __shared__ double red[3][8];
  double s[3] = {0.0, 0.0, 0.0};
  for (long long b = threadIdx.x; b < ncol; b += blockDim.x)
    for (int q = 0; q < 3; ++q) s[q] += partial[3 * b + q];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int q = 0; q < 3; ++q) {
    double v = s[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[3];
    for (int q = 0; q < 3; ++q) {
      t[q] = 0.0;
      for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) t[q] += red[q][ww];
    }
    out3[0] = 1.0 + sqrt_ra_pr * t[0] * vol;
    out3[1] = 0.5 * t[1] * vol;
    out3[2] = t[2] * vol;
  }
}

// Handle of the calling thread's current context (driver API cuCtxGetCurrent, reached through the
// runtime's entry-point query so that no driver library is linked), or null when unavailable.
using CtxGetCurrentFn = int (*)(void **);
void *current_context() {
  static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  void *ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array on the current device.  It is looked up once per device
// and context: a device reset (or any new context on the device) loads the module again, so the
// cached address is dropped when the current context handle differs from the one it was taken
// in.  Without a context handle the lookup runs on every call.
int scratch_for_current_device(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return AFID_E_CUDA;
  void *ctx = current_context();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      g_scratch_addr[dev] = nullptr;
      return AFID_E_CUDA;
    }
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_addr[dev];
  return AFID_OK;
}

}  // namespace

extern "C" int afid_gpu_globals_noalloc(int nxm, int nym, int nzm, int ldx, double alx3, double ra_pr,
                                        const double *vx, const double *vy, const double *vz,
                                        const double *temp, const double *g3rc, double *out3,
                                        void *stream) {
  if (nxm < 1 || nym < 1 || nzm < 1 || ldx < nxm + 1 || !(alx3 > 0.0) || !(ra_pr >= 0.0)) return AFID_E_INVALID;
  if (!vx || !vy || !vz || !temp || !g3rc || !out3) return AFID_E_INVALID;
  const long long ncol = (long long)nym * nzm;
  const long long need = (3 * ncol) * (long long)sizeof(double);
  if (need > (long long)AFID_NOALLOC_SCRATCH_BYTES) return AFID_E_CAPACITY;  // grid too large for the scratch
  void *scratch = nullptr;
  const int s = scratch_for_current_device(&scratch);
  if (s != AFID_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *partial = static_cast<double *>(scratch);
  const double dx = (double)nxm / alx3;
  const double vol = 1.0 / (alx3 * dx * (double)nzm * (double)nym);  // GlobalQuantities.F90:35
  const double sqrt_ra_pr = std::sqrt(ra_pr);
  // each launch reports its own status (cudaLaunchKernel's return value), so an error left
  // behind by the caller's earlier, unrelated CUDA calls is neither returned nor cleared here
  const dim3 grid1((unsigned)((ncol + 7) / 8)), block(256), one(1);
  void *a1[] = {&nxm, &nym, &nzm, &ldx, &vx, &vy, &vz, &temp, &g3rc, &partial};
  cudaError_t e = cudaLaunchKernel((const void *)k_noalloc_column_sums, grid1, block, a1, 0, st);
  if (e == cudaSuccess) {
    void *a2[] = {(void *)&partial, (void *)&ncol, (void *)&vol, (void *)&sqrt_ra_pr, (void *)&out3};
    e = cudaLaunchKernel((const void *)k_noalloc_finish, one, block, a2, 0, st);
  }
  return e == cudaSuccess ? AFID_OK : AFID_E_CUDA;
}
