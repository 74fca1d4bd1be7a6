// Scan kernels specialised for 0 value column(s) (see qm_scan_spec.cuh).
#define QM_SPEC_NV 0
#include "qm_scan_spec.cuh"
