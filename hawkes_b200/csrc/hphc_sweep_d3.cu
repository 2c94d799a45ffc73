// Pair-sweep kernels for D = 3 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 3
#include "hphc_sweep_dim.inc"
