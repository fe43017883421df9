// afid_k1_sal.cu — K1 instantiations that subtract the salinity buoyancy bycs * salc from the
// gravity component's explicit term (AddSalBuoyancy, salinity.F90:494-506), for contexts with
// an active salinity scalar (include/afid_salinity.h).  Kept apart so the plain instantiations
// carry no trace of it.
#include "afid_k1.cuh"

namespace afid {

cudaError_t launch_k1_fp64_sal(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  const bool two_d = (L.g.nzm == 1 || L.g.batch);
  return two_d ? launch_k1_T<double, true, true>(L, b, ns, var, ncol)
               : launch_k1_T<double, false, true>(L, b, ns, var, ncol);
}

cudaError_t launch_k1_mixed_sal(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  const bool two_d = (L.g.nzm == 1 || L.g.batch);
  return two_d ? launch_k1_T<float, true, true>(L, b, ns, var, ncol)
               : launch_k1_T<float, false, true>(L, b, ns, var, ncol);
}

}  // namespace afid
