// inst_f64_n0.cu -- instantiates every kernel for compute type double and e-e-n order 0
// (order 0 also serves nordc = 1, which has no e-e-n terms).
#include "launch.cuh"

CHAMP_INST(f64, double, 0)
