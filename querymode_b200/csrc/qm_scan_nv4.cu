// Scan kernels specialised for 4 value column(s) (see qm_scan_spec.cuh).
#define QM_SPEC_NV 4
#include "qm_scan_spec.cuh"
