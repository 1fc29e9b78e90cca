// Fused chain kernels for 2048-point A-scans.
#define OPE_CHAIN_N 2048
#include "chain_inst.cuh"
