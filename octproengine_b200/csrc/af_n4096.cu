// Autofocus kernels for 4096-point A-scans.
#define OPE_AF_N 4096
#include "af_inst.cuh"
