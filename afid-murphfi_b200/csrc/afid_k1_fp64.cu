// afid_k1_fp64.cu — K1 instantiations with FP64 explicit terms and RK3 histories.
#include "afid_k1.cuh"

namespace afid {

cudaError_t launch_k1_fp64(const LaunchCtx &L, const SubstepBuffers &b, int ns, int var, int ncol) {
  if (L.g.salc) return launch_k1_fp64_sal(L, b, ns, var, ncol);
  const bool two_d = (L.g.nzm == 1 || L.g.batch);  // z neighbours are the column itself
  return two_d ? launch_k1_T<double, true, false>(L, b, ns, var, ncol)
               : launch_k1_T<double, false, false>(L, b, ns, var, ncol);
}

int k1_shapes(int M, int *tpc, int *rpt, int *cap, int *pol) {
  const int mi = k1_m_index(M);
  static_assert(kK1MaxShapes <= AFID_TUNE_MAX, "the tune record must hold every K1 shape");
  for (int v = 0; v < kK1ShapeCount[mi]; ++v) {
    if (tpc) tpc[v] = kK1Shapes[mi][v].tpc;
    if (rpt) rpt[v] = kK1Shapes[mi][v].rpt;
    if (cap) cap[v] = kK1Shapes[mi][v].cap;
    // reported policy: bit 0 cache hints, bit 1 two columns per block, bit 2 adjacent rows,
    // bit 3 the persistent kernel with its tables in shared memory, bit 4 the first row's table
    // operands loaded before the staging wait, bit 5 the solves' forward factors loaded before
    // the barrier that precedes them
    if (pol)
      pol[v] = (kK1Shapes[mi][v].pol & 5) | (kK1Shapes[mi][v].ny == 2 ? 2 : 0) | (kK1Shapes[mi][v].ny == 0 ? 8 : 0) |
               ((kK1Shapes[mi][v].pol & 8) ? 16 : 0) | ((kK1Shapes[mi][v].pol & 16) ? 32 : 0);
  }
  return kK1ShapeCount[mi];
}

bool k1_shape_usable(int M, int v, bool batch, bool two_d) {
  const int mi = k1_m_index(M);
  if (v < 0 || v >= kK1ShapeCount[mi]) return false;
  const K1Shape &s = kK1Shapes[mi][v];
  if (batch && s.ny == 0) return false;
  if (s.ny == 0 && k1p_groups(M, two_d) < 2) return false;
  return true;
}

}  // namespace afid
