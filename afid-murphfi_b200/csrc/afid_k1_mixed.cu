// afid_k1_mixed.cu — K1 instantiations with FP32 explicit terms and RK3 histories (FP64 state, RHS and solves).
#include "afid_k1.cuh"

namespace afid {

cudaError_t launch_k1_mixed(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  if (L.g.salc) return launch_k1_mixed_sal(L, b, ns, var, ncol);
  const bool two_d = (L.g.nzm == 1 || L.g.batch);  // z neighbours are the column itself
  return two_d ? launch_k1_T<float, true, false>(L, b, ns, var, ncol)
               : launch_k1_T<float, false, false>(L, b, ns, var, ncol);
}

}  // namespace afid
