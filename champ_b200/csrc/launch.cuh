// launch.cuh -- kernel dispatch over (precision, e-e-n order, multi-determinant).
#pragma once
#include "ctx.h"

#define fail champ_fail
// ---- kernel dispatch over (precision, e-e-n order)
template <class K>
static int set_attrs(champ_ctx *c, K kern) {
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem));
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
  return CHAMP_OK;
}
template <class T, int NORD, bool MD>
static int set_smem_attrs(champ_ctx *c) {
  int rc = set_attrs(c, k_eval<T, NORD, MD>);
  if (!rc) rc = set_attrs(c, k_propose<T, NORD, MD>);
  if (!rc) rc = set_attrs(c, k_accept<T, MD>);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD>);
  if (!rc) rc = set_attrs(c, k_dmc_move<T, NORD, MD>);
  if (!rc) {
    CK(cudaFuncSetAttribute(k_pgrad<T, NORD, MD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_pg));
    CK(cudaFuncSetAttribute(k_pgrad<T, NORD, MD>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            (int)cudaSharedmemCarveoutMaxShared));
  }
  return rc;
}

template <class T, int NORD, bool MD>
static int launch_t(champ_ctx *c, Op op, const OpArgs &a) {
  Sys<T> &s = sysof<T>(c);
  State<T> st = a.st_override ? *(const State<T> *)a.st_override : stof<T>(c);
  st.W = a.st_override ? a.nw_override : c->W;
  dim3 grid((st.W + c->wpb - 1) / c->wpb), block(32 * c->wpb);
  const double *R = c->rot;
  switch (op) {
  case Op::Eval:
  case Op::EvalOut:
    k_eval<T, NORD, MD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7], R[8],
                                                       op == Op::EvalOut ? 1 : 0);
    break;
  case Op::Propose:
  case Op::ProposeGrad:
    k_propose<T, NORD, MD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.e, a.xnew, a.ratio, op == Op::ProposeGrad ? a.grad : nullptr);
    break;
  case Op::Accept:
    k_accept<T, MD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.e, a.mask);
    break;
  case Op::PGrad:
    k_pgrad<T, NORD, MD><<<dim3((c->W + c->wpb_pg - 1) / c->wpb_pg), dim3(32 * c->wpb_pg), c->smem_pg, c->stream>>>(s, st, c->lay, a.pgout, R[0], R[1], R[2], R[3], R[4],
                                                                 R[5], R[6], R[7], R[8]);
    break;
  case Op::DmcMove:
    k_dmc_move<T, NORD, MD><<<dim3((c->dpar.wmax + c->wpb - 1) / c->wpb), block, c->smem, c->stream>>>(
        s, st, c->lay, c->dpar, c->dA, a.istep);
    break;
  case Op::DmcCopy: {
    k_dmc_copy<T><<<592, 128, 0, c->stream>>>(st, st2of<T>(c), c->dA, c->dB, c->N, c->C, c->dpar.wmax);
    break;
  }
  case Op::Vmc:
    k_vmc<T, NORD, MD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.nsweep, a.seed, a.sweep0, a.step);
    break;
  }
  CK(cudaGetLastError());
  return CHAMP_OK;
}

template <class T, bool MD>
static int launch_m(champ_ctx *c, Op op, const OpArgs &a) {
  switch (c->nordc) {
  case 0: case 1: return launch_t<T, 0, MD>(c, op, a);
  case 4: return launch_t<T, 4, MD>(c, op, a);
  case 5: return launch_t<T, 5, MD>(c, op, a);
  default: return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
template <class T>
static int launch_p(champ_ctx *c, Op op, const OpArgs &a) {
  return c->md.multidet ? launch_m<T, true>(c, op, a) : launch_m<T, false>(c, op, a);
}

template <class T, bool MD>
static int attrs_m(champ_ctx *c) {
  switch (c->nordc) {
  case 0: case 1: return set_smem_attrs<T, 0, MD>(c);
  case 4: return set_smem_attrs<T, 4, MD>(c);
  case 5: return set_smem_attrs<T, 5, MD>(c);
  default: return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
template <class T>
static int attrs_p(champ_ctx *c) {
  return c->md.multidet ? attrs_m<T, true>(c) : attrs_m<T, false>(c);
}

#undef fail
