// Pair-sweep kernels for D = 5 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 5
#include "hphc_sweep_dim.inc"
