// afid_internal.h — declarations shared by the kernel and API translation units.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "afid_device.cuh"

namespace afid {

// Everything a launcher needs that does not change between substeps.
struct LaunchCtx {
  Geom g;
  Tables t;
  cudaStream_t stream;
  int M;           // rows per lane of the partitioned x-solves (32*M >= nxm)
  bool mixed;      // FP32 explicit terms / transforms
  int tx_y, tx_z;  // x-tile widths of the shared-memory (fallback) FFT kernels
  bool warp_fft;   // register-resident warp FFT when N = 32*{1,2,3,4,6,8,12,16,24,32}
  int k1_var;      // K1 thread shape (index into the shapes of k1_shapes(M)), set by the autotuner
  int k4_var;      // K4 form: 0 one mode a warp, 1 persistent with the next mode prefetched (FP64)
  int fftz_var;    // z transforms (K3/K5): 0 a tile a block, 1 persistent with the next tile
                   // prefetched, 2 the same with tensor copies (FP64)
  int ify_var;     // inverse y transform (K6): 0 per-thread copies, 1 tensor copies (FP64 single domain)
  int div_var;     // divergence + forward y transform (K2): 0 per-thread loads, 1 tensor copies (FP64
                   // single domain)
  FftPlan plan_y, plan_z;
  const void *twy, *twz;  // twiddle tables (double2 or float2)
};

// Buffers of one substep.  K1 reads the state (vx, vy, vz, temp, pr) and writes the
// intermediate fields (*_o); the pressure kernels read the intermediate velocities and write
// the projected velocities back into the state arrays.
struct SubstepBuffers {
  const StepCoef *sc;
  const double *cn_tab;
  double *vx, *vy, *vz, *temp, *pr;
  void *rux, *ruy, *ruz, *rut;  // double or float (mixed)
  double *vx_o, *vy_o, *vz_o, *temp_o;
  void *spec;                   // complex spectrum (double2 or float2)
  void *phi;                    // pressure correction (double or float)
  int *err;
  // K2 input: nullptr = the divergence of (vx_o, vy_o, vz_o); else this field (spectra)
  const double *fft_field = nullptr;
};

struct CnInputs {
  int nmat = 3;  // matrices per substep: vx, vy/vz, temp (3), or one temperature-like matrix (1)
  const double *am[3], *ac[3], *ap[3];
  int off[3], n[3];
  double al[3], ga[3], ro[3];
  double dt, beta, pect, ren;
  int ns0, nsub, M;
  double *tab;
  StepCoef *sc;
  // batch mode (else nullptr / 0): per-instance dt on the device, scalars, active flags
  const double *dt_dev = nullptr;
  const InstScal *inst = nullptr;
  const unsigned char *active = nullptr;
  int ninst = 0;
};

int cn_choose_M(int nxm);
// Dynamic shared memory of the fused explicit/implicit kernel (29 staged x-columns + solve rows).
size_t k1_smem_bytes(int ldx, int M, bool mixed, bool two_d);
size_t cn_tab_doubles(int M, int nsst);
cudaError_t launch_cn_tables(const LaunchCtx &L, const CnInputs &in);
cudaError_t launch_explicit_implicit(const LaunchCtx &L, const SubstepBuffers &b, int ns);
// K1 over the first ncol columns with thread shape `var` (autotuner samples use ncol < all).
cudaError_t launch_k1_fp64(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol);
cudaError_t launch_k1_mixed(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol);
// The same with the salinity buoyancy in the explicit terms (L.g.salc set).
cudaError_t launch_k1_fp64_sal(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol);
cudaError_t launch_k1_mixed_sal(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol);
// Thread shapes of K1 for M: fills tpc[]/rpt[]/cap[]/pol[] (up to AFID_TUNE_MAX) and returns their number.
int k1_shapes(int M, int *tpc, int *rpt, int *cap, int *pol);
// Whether K1 shape v of this M can run on a context (the forms that keep one substep's CN
// factors per block do not take a batch, whose factors differ per instance).
bool k1_shape_usable(int M, int v, bool batch, bool two_d);
// The kernels of one substep, in launch order (K1 .. K7).
enum class Stage { ExplicitImplicit = 0, DivFftY, FftZFwd, Tridiag, FftZInv, IfftY, Correct };
constexpr int kNumStages = 7;
cudaError_t launch_stage(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st);
cudaError_t launch_max_reduce(const LaunchCtx &L, bool div, const double *vx, const double *vy,
                              const double *vz, unsigned long long *out);
cudaError_t launch_globals(const LaunchCtx &L, const double *vx, const double *vy,
                           const double *vz, const double *temp, double *partial, double *out3);
int globals_partial_blocks(const Geom &g);

// ---- multi-resolution salinity (afid_salinity.cu) ----------------------------------------
struct SalGeom {
  int nxmr, nymr, nzmr, ldr;       // refined cells and x stride (>= nxmr + 1, multiple of 8)
  int ldu;                         // x stride of wall-extended refined columns (>= nxmr + 4)
  int MR;                          // rows per lane of the refined CN solve (32 MR >= nxmr)
  double dxr, dyr, dzr;
  double udyr, udzr;               // 0.5 dyr, 0.5 dzr        (ExplicitSalinity advection)
  double udyrq, udzrq;             // dyr^2/pecs, dzr^2/pecs  (ExplicitSalinity diffusion)
  double lya, lza;                 // 1/dyr, 1/dzr            (InterpVelMgrd integration)
  double pecs;
  int sfixs, sfixn;
};
struct SalTables {
  const double *lxa;               // [nxmr] xcr(k+1) - xcr(k)
  const double *udx3mr, *tdxr;     // [nxmr] dxr/d3xcr, 0.5 dxr/g3rmr
  const double *ap, *ac, *am;      // [nxmr] ap3sskr, ac3sskr, am3sskr
  const double *salbp, *saltp;     // [nymr*nzmr]
  const int *st[6];                // to_ref x, y, z; to_coarse x, y, z: first source row
  const double *w[6];              //   and the 4 weights of every target
};
struct SalCtx {
  SalGeom sg{};
  SalTables st{};
  int active_s = 0;
  double bycs = 0.0;
  size_t relems = 0;               // elements of one refined field
  double *sal = nullptr, *sal_o = nullptr, *rusal = nullptr;
  double *vxr = nullptr, *vyr = nullptr, *vzr = nullptr;
  double *gyr = nullptr, *gzr = nullptr;         // refined y/z velocity gradients (scratch)
  double *tmp = nullptr;                         // z-contracted interpolation passes (scratch)
  double *gx = nullptr, *gy = nullptr, *gz = nullptr, *salc = nullptr;  // coarse
  double *cn_tab = nullptr;
  StepCoef *sc = nullptr;
  double *partial = nullptr, *prof_out = nullptr;
  int prof_blocks = 0;
  unsigned long long *red = nullptr;
  int *err = nullptr;                            // the context's error word
  const double *am_d = nullptr, *ac_d = nullptr, *ap_d = nullptr;
};
// ExplicitSalinity + ImplicitSalinity + SolveImpEqnUpdate_Sal: sal -> sal_o, rusal in place.
cudaError_t launch_sal_step(const LaunchCtx &L, const SalCtx &S, int ns);
// InterpVelMgrd + InterpSalMultigrid from the state (vx, vy, vz) and S.sal.
cudaError_t launch_sal_interp(const LaunchCtx &L, const SalCtx &S, const double *vx, const double *vy,
                              const double *vz);
cudaError_t launch_sal_cfl(const LaunchCtx &L, const SalCtx &S);
// Six profiles (Sbar, Srms, vxS, vyS, vzS, chiS) into out[6 * nxmr] (device).
cudaError_t launch_sal_profiles(const LaunchCtx &L, const SalCtx &S, double *out);
int sal_prof_blocks(const SalGeom &sg);
size_t sal_step_smem_bytes(int MR, bool two_d);
constexpr int kSalLaunchesInterp = 7;
cudaError_t launch_repack(cudaStream_t st, const double *src, int sld, double *dst, int dld, int width,
                          size_t rows);

}  // namespace afid

#include "afid_gpu.h"

// The context behind afid_ctx_t (include/afid_gpu.h).
struct afid_ctx {
  int dev = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaError_t last_cuda = cudaSuccess;
  long long launches = 0;
  int nsst = 3;
  double alx3 = 1.0;
  afid::LaunchCtx L{};
  // device allocations
  std::vector<void *> allocs;
  long long dev_bytes = 0;  // sum of the allocations above
  double *vx = nullptr, *vy = nullptr, *vz = nullptr, *temp = nullptr, *pr = nullptr;
  double *vx_o = nullptr, *vy_o = nullptr, *vz_o = nullptr, *temp_o = nullptr;
  void *rux = nullptr, *ruy = nullptr, *ruz = nullptr, *rut = nullptr;
  void *spec = nullptr, *phi = nullptr;
  double *cn_tab = nullptr;
  afid::StepCoef *sc = nullptr;
  int *err = nullptr;
  unsigned long long *red = nullptr;
  double *partial = nullptr, *gsum = nullptr;
  double *host_scratch = nullptr;  // pinned, 8 doubles
  // device tables for the CN builder
  const double *am[3], *ac[3], *ap[3];
  size_t field_elems = 0;
  // optional per-kernel event timing
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Rec { int cls; size_t a, b; };
  std::vector<Rec> recs;
  // scratch of the profile reductions (afid_stats.cu), allocated on first use
  double *stats_buf = nullptr;
  size_t stats_elems = 0;
  // spectra accumulators (vx, vy, vz, temp; nxm x nyh x nzm each) and the averaged interval
  double *spec_acc = nullptr;
  double spec_tav = 0.0;
  // K1 thread-shape autotuner
  bool tuned = false;
  afid_tune_info_t tune{};
  // batch mode: instance scalars and active flags on the device (see afid::BatchSpec)
  int ninst = 0;
  afid::InstScal *inst_dev = nullptr;
  unsigned char *active_dev = nullptr;
  // multi-resolution salinity (include/afid_salinity.h), nullptr when off
  afid::SalCtx *sal = nullptr;
};

namespace afid {

// A batch of independent 2-D instances of one size class, stacked along z (Geom::batch).
struct BatchSpec {
  int ninst;
  const InstScal *inst;   // [ninst] host
  const double *ak2;      // [ninst * nym] host, per-instance modified wavenumbers in y
  const double *tempbp;   // [ninst * nym] host plate values
  const double *temptp;
};

int ctx_create(const afid_grid_t *grid, const afid_params_t *prm, const BatchSpec *bs, afid_ctx_t **out);
SubstepBuffers ctx_buffers(afid_ctx_t *ctx);
int ctx_run_substep(afid_ctx_t *ctx, int ns);
int ctx_build_cn_batch(afid_ctx_t *ctx, const double *dt_dev);
int ctx_fail(afid_ctx_t *ctx, cudaError_t e);
int ctx_update_params(afid_ctx_t *ctx, const afid_grid_t *grid, const afid_params_t *prm);
int ctx_autotune(afid_ctx_t *ctx, bool force);
int ctx_mean_profiles(afid_ctx_t *ctx, int col0, int ncols, double ny_nz, double ren, double pect, double *out);

}  // namespace afid

