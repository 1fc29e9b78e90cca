// Autofocus kernels for 1024-point A-scans.
#define OPE_AF_N 1024
#include "af_inst.cuh"
