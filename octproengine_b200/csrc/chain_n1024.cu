// Fused chain kernels for 1024-point A-scans.
#define OPE_CHAIN_N 1024
#include "chain_inst.cuh"
