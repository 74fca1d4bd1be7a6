// qm_scan_spec.cuh — instantiations of the scan kernel for one value-column
// count (QM_SPEC_NV, defined by the including qm_scan_nv*.cu): every
// dedupe flag x key kind combination the planner produces, plus their
// shared-memory attribute setter and launcher.
#include "qm_scan.cuh"

#define QM_PASTE2(a, b) a##b
#define QM_PASTE(a, b) QM_PASTE2(a, b)
#define QM_SPEC_FN(x) QM_PASTE(QM_PASTE(qm_scan_nv, QM_SPEC_NV), x)

// (dedupe, key kind) pairs: the no-GROUP-BY plan always deduplicates
#define QM_SPEC_PAIRS(X) \
  X(0, QM_KK_ANY) X(0, QM_KK_I64) X(0, QM_KK_I32) X(1, QM_KK_ANY) X(1, QM_KK_I64) X(1, QM_KK_I32) X(1, QM_KK_NONE)

cudaError_t QM_SPEC_FN(_attr)(int max_smem) {
  using namespace qm;
  cudaError_t e = cudaSuccess;
#define QM_ATTR_(DD, KK)                                                                            \
  if (e == cudaSuccess)                                                                             \
    e = cudaFuncSetAttribute(qm_scan_kernel<false, false, DD, QM_SPEC_NV, KK>,                      \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  QM_SPEC_PAIRS(QM_ATTR_)
#undef QM_ATTR_
  return e;
}

cudaError_t QM_SPEC_FN(_launch)(const qm_scan_args &a, int dd, int kk, int blocks, size_t smem, cudaStream_t st) {
  using namespace qm;
#define QM_LAUNCH_(DD, KK)                                                                  \
  if (dd == DD && kk == KK) {                                                               \
    qm_scan_kernel<false, false, DD, QM_SPEC_NV, KK><<<blocks, QM_SCAN_THREADS, smem, st>>>(a); \
    return cudaGetLastError();                                                              \
  }
  QM_SPEC_PAIRS(QM_LAUNCH_)
#undef QM_LAUNCH_
  return cudaErrorInvalidValue;
}
