// inst_f64_n4.cu -- instantiates every kernel for compute type double and e-e-n order 4
// (order 0 also serves nordc = 1, which has no e-e-n terms).
#include "launch.cuh"

CHAMP_INST(f64, double, 4)
