// nbl_trav_count32r.cu -- the FP32-filter count pass for work items that
// may be runs of several home cells (the instantiations with RUN = true).
#define NBL_TRAV_RUNS 1
#include "nbl_trav_count32.cu"
