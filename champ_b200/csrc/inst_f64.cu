// inst_f64.cu -- instantiates every kernel for compute type double.
#include "launch.cuh"

int launch_f64(champ_ctx *c, Op op, const OpArgs &a) { return launch_p<double>(c, op, a); }
int attrs_f64(champ_ctx *c) { return attrs_p<double>(c); }
