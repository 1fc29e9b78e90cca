// Fused chain kernels for 4096-point A-scans.
#define OPE_CHAIN_N 4096
#include "chain_inst.cuh"
