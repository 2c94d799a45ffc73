// Pair-sweep kernels for D = 6 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 6
#include "hphc_sweep_dim.inc"
