// Scan kernels specialised for 3 value column(s) (see qm_scan_spec.cuh).
#define QM_SPEC_NV 3
#include "qm_scan_spec.cuh"
