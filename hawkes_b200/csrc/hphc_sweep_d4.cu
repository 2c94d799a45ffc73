// Pair-sweep kernels for D = 4 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 4
#include "hphc_sweep_dim.inc"
