// Fused chain kernels for 512-point A-scans.
#define OPE_CHAIN_N 512
#include "chain_inst.cuh"
