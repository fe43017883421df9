// afid_internal.h — declarations shared by the kernel and API translation units.
#pragma once
#include <cuda_runtime.h>

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
};

struct CnInputs {
  const double *am[3], *ac[3], *ap[3];
  int off[3], n[3];
  double al[3], ga[3], ro[3];
  double dt, beta, pect, ren;
  int ns0, nsub, M;
  double *tab;
  StepCoef *sc;
};

int cn_choose_M(int nxm);
size_t cn_tab_doubles(int M, int nsst);
cudaError_t launch_cn_tables(const LaunchCtx &L, const CnInputs &in);
cudaError_t launch_explicit_implicit(const LaunchCtx &L, const SubstepBuffers &b, int ns);
// The kernels of one substep, in launch order (K1 .. K7).
enum class Stage { ExplicitImplicit = 0, DivFftY, FftZFwd, Tridiag, FftZInv, IfftY, Correct };
constexpr int kNumStages = 7;
cudaError_t launch_stage(const LaunchCtx &L, const SubstepBuffers &b, int ns, Stage st);
cudaError_t launch_max_reduce(const LaunchCtx &L, bool div, const double *vx, const double *vy,
                              const double *vz, unsigned long long *out);
cudaError_t launch_globals(const LaunchCtx &L, const double *vx, const double *vy,
                           const double *vz, const double *temp, double *partial, double *out3);
int globals_partial_blocks(const Geom &g);

}  // namespace afid
