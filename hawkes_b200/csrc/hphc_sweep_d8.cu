// Pair-sweep kernels for D = 8 (see hphc_sweep.cuh).
#define HPHC_SWEEP_DIM 8
#include "hphc_sweep_dim.inc"
