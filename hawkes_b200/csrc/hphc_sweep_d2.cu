// Pair-sweep kernels for D = 2 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 2
#include "hphc_sweep_dim.inc"
