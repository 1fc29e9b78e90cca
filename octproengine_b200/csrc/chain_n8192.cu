// Fused chain kernels for 8192-point A-scans.
#define OPE_CHAIN_N 8192
#include "chain_inst.cuh"
