// nbl_trav_fill32r.cu -- the fill pass after the FP32-filter count for work
// items that may be runs of several home cells (RUN = true).
#define NBL_TRAV_RUNS 1
#include "nbl_trav_fill32.cu"
