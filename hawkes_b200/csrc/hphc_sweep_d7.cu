// Pair-sweep kernels for D = 7 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 7
#include "hphc_sweep_dim.inc"
