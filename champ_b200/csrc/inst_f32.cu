// inst_f32.cu -- instantiates every kernel for compute type float.
#include "launch.cuh"

int launch_f32(champ_ctx *c, Op op, const OpArgs &a) { return launch_p<float>(c, op, a); }
int attrs_f32(champ_ctx *c) { return attrs_p<float>(c); }
