// Autofocus kernels for 2048-point A-scans.
#define OPE_AF_N 2048
#include "af_inst.cuh"
