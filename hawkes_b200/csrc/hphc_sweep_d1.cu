// Pair-sweep kernels for D = 1 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 1
#include "hphc_sweep_dim.inc"
