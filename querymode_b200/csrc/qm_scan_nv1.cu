// Scan kernels specialised for 1 value column(s) (see qm_scan_spec.cuh).
#define QM_SPEC_NV 1
#include "qm_scan_spec.cuh"
