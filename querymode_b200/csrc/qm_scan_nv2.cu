// Scan kernels specialised for 2 value column(s) (see qm_scan_spec.cuh).
#define QM_SPEC_NV 2
#include "qm_scan_spec.cuh"
