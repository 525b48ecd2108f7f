// inst_f32_n4.cu -- instantiates every kernel for compute type float and e-e-n order 4
// (order 0 also serves nordc = 1, which has no e-e-n terms).
#include "launch.cuh"

CHAMP_INST(f32, float, 4)
