// launch.cuh -- kernel dispatch over (precision, e-e-n order, multi-determinant).
#pragma once
#include <algorithm>
#include <type_traits>

#include "ctx.h"

#define fail champ_fail
// ---- kernel dispatch over (precision, e-e-n order)
template <class K>
static int set_attrs(champ_ctx *c, K kern, size_t smem) {
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
  return CHAMP_OK;
}
template <class T, int NORD, bool MD>
static int set_smem_attrs(champ_ctx *c) {
  const size_t sm = kcfg<T>(c).smem;
  int rc = set_attrs(c, k_eval<T, NORD, MD>, sm);
  if (!rc) rc = set_attrs(c, k_propose<T, NORD, MD>, sm);
  if (!rc) rc = set_attrs(c, k_accept<T, MD>, sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 0>, sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 1>, std::is_same<T, float>::value ? std::max(sm, c->kfm.smem) : sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 2>, sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 3>, sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 0, 6>, sm);
  if (!rc) rc = set_attrs(c, k_vmc<T, NORD, MD, 1, 6>, sm);
  if (!rc) rc = set_attrs(c, k_dmc_move<T, NORD, MD>, sm);
  if (!rc) rc = set_attrs(c, k_dmc_tmove<T, NORD, MD>, sm);
  if (!rc && std::is_same<T, float>::value && c->prec == CHAMP_PREC_FP32) {
    CK(cudaFuncSetAttribute(orbtc::k_orb_tc<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024 + 128));
    CK(cudaFuncSetAttribute(orbtc::k_orb_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024 + 128));
    CK(cudaFuncSetAttribute(orbtc::k_orb_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)orbtc::smem_bytes(256, 2)));
    CK(cudaFuncSetAttribute(orbf::k_orb_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)orbf::fsmem_bytes(96)));
    CK(cudaFuncSetAttribute(k_basis_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)std::min<size_t>(4 * (size_t)c->nbasis * 5 * sizeof(float), 227 * 1024)));
  }
  if (!rc && c->el_staged && std::is_same<T, double>::value) {
    rc = set_attrs(c, k_el_jas<T, NORD>, c->el_smem[0]);
    if (!rc) rc = set_attrs(c, k_el_jas<T, NORD, true>, c->el_smem[0]);
    if (!rc) rc = set_attrs(c, k_el_orb<T>, c->el_smem[1]);
    if (!rc) rc = set_attrs(c, k_el_fin<T, NORD, MD>, c->el_smem[2]);
    if (!rc) rc = set_attrs(c, k_el_inv, sizeof(double) * CHAMP_MAX_SPIN * CHAMP_MAX_SPIN);
  }
  if (!rc && c->smem_pg > 0) {
    for (auto kern : {k_pgrad<T, NORD, MD, 1>, k_pgrad<T, NORD, MD, 2>, k_pgrad<T, NORD, MD, 3>, k_pgrad<T, NORD, MD, 4>}) {
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_pg));
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
    }
  }
  return rc;
}

// Orbitals (5 channels) of every electron of every walker in st.orb5 by the tensor cores:
// basis rows to HBM, then one tcgen05 contraction per spin.
template <class T>
static int run_orb_tc(champ_ctx *c, const State<T> &st) {
  if constexpr (!std::is_same<T, float>::value) {
    return fail(CHAMP_EINVAL, "tensor-core orbitals are a mixed-precision path");
  } else {
    const int sm = c->num_sms > 0 ? c->num_sms : 148;
    if (c->tc_mode == 1) {
      for (int sp = 0; sp < 2; sp++) {
        const int n = sp ? c->ndn : c->nup;
        if (n == 0) continue;
        orbf::FArgs f;
        f.x = st.x;
        f.bhi = c->tc_bf[sp][0];
        f.blo = c->tc_bf[sp][1];
        f.blk_sh = c->tc_blk_sh;
        f.kpos = c->tc_kpos;
        f.orb = st.orb5;
        f.M = st.W * n;
        f.Kq = c->tc_kq;
        f.nkb = c->tc_nkb;
        f.Np = c->tc_Np[sp];
        f.ncols = c->tc_fcols[sp];
        f.n = n;
        f.N = c->N;
        f.e0 = sp ? c->nup : 0;
        f.nomax = c->nomax;
        f.nocc = c->md.nocc[sp];
        f.kchunk = c->tc_kchunk > 0 ? c->tc_kchunk : f.nkb;
        f.err = c->tc_err;
        const int tiles = (f.M + orbtc::BM - 1) / orbtc::BM;
        orbf::k_orb_fused<<<(unsigned)std::min(tiles, sm), orbf::NTF, orbf::fsmem_bytes(f.Np), c->stream>>>(c->sf, f);
        CK(cudaGetLastError());
      }
      return CHAMP_OK;
    }
    const long long items = (long long)st.W * c->N;
    long long gb = std::min<long long>((items + 3) / 4, (long long)sm * 8);
    k_basis_rows<<<(unsigned)std::max<long long>(gb, 1), 128, 4 * (size_t)c->nbasis * 5 * sizeof(float), c->stream>>>(
        c->sf, st.x, items, c->tc_Kp, c->tc_phi);
    CK(cudaGetLastError());
    for (int sp = 0; sp < 2; sp++) {
      const int n = sp ? c->ndn : c->nup;
      if (n == 0) continue;
      orbtc::Args g;
      g.phi = c->tc_phi;
      g.bhi = c->tc_b[sp][0];
      g.blo = c->tc_b[sp][1];
      g.orb = st.orb5;
      g.M = st.W * n * 5;
      g.Kp = c->tc_Kp;
      g.Np = c->tc_Np[sp];
      g.ncols = c->tc_ncols[sp];
      g.n = n;
      g.N = c->N;
      g.e0 = sp ? c->nup : 0;
      g.nomax = c->nomax;
      g.nocc = c->md.nocc[sp];
      // the same MMA chain length as the fused kernel's chunks (its K-blocks are half as long)
      g.kchunk = c->tc_kchunk > 0 ? std::max(1, c->tc_kchunk * orbf::BKF / orbtc::BK) : g.Kp / orbtc::BK;
      g.err = c->tc_err;
      const int tiles = (g.M + orbtc::BM - 1) / orbtc::BM, ns = orbtc::stages_for(g.Np);
      const unsigned grid = (unsigned)std::min(tiles, sm);
      const size_t smb = orbtc::smem_bytes(g.Np, ns);
      if (ns == 4) orbtc::k_orb_tc<4><<<grid, orbtc::NTHR, smb, c->stream>>>(g);
      else if (ns == 3) orbtc::k_orb_tc<3><<<grid, orbtc::NTHR, smb, c->stream>>>(g);
      else orbtc::k_orb_tc<2><<<grid, orbtc::NTHR, smb, c->stream>>>(g);
      CK(cudaGetLastError());
    }
    return CHAMP_OK;
  }
}

// The full evaluation of every walker as the four parts of elstage.cuh (FP64 state in HBM).
template <class T, int NORD, bool MD>
static int run_el_staged(champ_ctx *c, const State<T> &st, bool outputs, bool stats, const ElRot &rot,
                         bool rebuild = false) {
  if constexpr (!std::is_same<T, double>::value) {
    return fail(CHAMP_EINVAL, "internal: the staged evaluation is an FP64 path");
  } else {
    Sys<T> &s = sysof<T>(c);
    const int W = st.W, sm = c->num_sms > 0 ? c->num_sms : 148;
    const int w0 = c->el_wpb[0], w1 = c->el_wpb[1], w2 = c->el_wpb[2];
    const bool vo = rebuild && !outputs && !stats;  // the moves' state only: no velocities, no E_L
    if (vo) k_el_jas<T, NORD, true><<<(W + w0 - 1) / w0, 32 * w0, c->el_smem[0], c->stream>>>(s, st);
    else k_el_jas<T, NORD><<<(W + w0 - 1) / w0, 32 * w0, c->el_smem[0], c->stream>>>(s, st);
    CK(cudaGetLastError());
    const long long items = (long long)W * c->N;
    const long long g1 = std::min<long long>((items + w1 - 1) / w1, (long long)sm * 64);
    k_el_orb<T><<<(unsigned)std::max<long long>(g1, 1), 32 * w1, c->el_smem[1], c->stream>>>(
        s, st, c->orb_coop && c->orb_coop_ok, c->orb_stage);
    CK(cudaGetLastError());
    const int nmax = std::max(c->nup, c->ndn);
    k_el_inv<<<2 * W, 128, sizeof(double) * nmax * nmax, c->stream>>>(st.ainv, st.astride, c->nup, c->ndn, W, st.el_sc);
    CK(cudaGetLastError());
    k_el_fin<T, NORD, MD><<<(W + w2 - 1) / w2, 32 * w2, c->el_smem[2], c->stream>>>(
        s, st, c->el_nscr, outputs ? 1 : 0, stats ? 1 : 0, rot, vo ? 1 : 0);
    CK(cudaGetLastError());
    c->orb5_valid = st.orb5 == c->std_.orb5;  // k_el_orb wrote every electron's row
    return CHAMP_OK;
  }
}

template <class T, int NORD, bool MD>
static int launch_t(champ_ctx *c, Op op, const OpArgs &a) {
  Sys<T> &s = sysof<T>(c);
  State<T> st = a.st_override ? *(const State<T> *)a.st_override : stof<T>(c);
  st.W = a.st_override ? a.nw_override : c->W;
  const KCfg &K = kcfg<T>(c);
  dim3 grid((st.W + K.wpb - 1) / K.wpb), block(32 * K.wpb);
  // the FP64 state's orbital rows stay current only through evaluations and the accelerated
  // mover's sweeps, which update them (run_el_staged marks them current)
  if (op != Op::Eval && op != Op::EvalOut && op != Op::Vmc) c->orb5_valid = false;
  const double *R = c->rot;
  switch (op) {
  case Op::Eval:
  case Op::EvalOut: {
    const bool tc = c->tc_on && !a.st_override;  // only FP32 contexts turn it on
    if (c->el_staged && std::is_same<T, double>::value && !a.st_override) {
      ElRot rot{};
      for (int i = 0; i < 9; i++) rot.R[i] = R[i];
      return run_el_staged<T, NORD, MD>(c, st, op == Op::EvalOut, false, rot, a.rebuild);
    }
    c->orb5_valid = false;
    if (tc) {
      int rc = run_orb_tc<T>(c, st);
      if (rc) return rc;
    }
    k_eval<T, NORD, MD><<<grid, block, K.smem, c->stream>>>(s, st, K.lay, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7], R[8],
                                                       op == Op::EvalOut ? 1 : 0, tc ? 1 : 0);
    break;
  }
  case Op::Propose:
  case Op::ProposeGrad:
    k_propose<T, NORD, MD><<<grid, block, K.smem, c->stream>>>(s, st, K.lay, a.e, a.xnew, a.ratio, op == Op::ProposeGrad ? a.grad : nullptr);
    break;
  case Op::Accept:
    k_accept<T, MD><<<grid, block, K.smem, c->stream>>>(s, st, K.lay, a.e, a.mask);
    break;
  case Op::PGrad:
  case Op::PGradBwd: {
    const dim3 pgrid((c->W + c->wpb_pg - 1) / c->wpb_pg), pblock(32 * c->wpb_pg);
    auto kern = a.pgout.part == 1 ? k_pgrad<T, NORD, MD, 1>
              : a.pgout.part == 2 ? k_pgrad<T, NORD, MD, 2>
              : a.pgout.part == 3 ? k_pgrad<T, NORD, MD, 3> : k_pgrad<T, NORD, MD, 4>;
    kern<<<pgrid, pblock, c->smem_pg, c->stream>>>(s, st, K.lay, a.pgout, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7], R[8]);
    break;
  }
  case Op::DmcMove: {
    // persistent: as many blocks as the SMs can hold at once (at most 16 per SM; a block that
    // finds the work counter exhausted exits at once), no more than the walkers need
    const int sm = c->num_sms > 0 ? c->num_sms : 148;
    const int need = (c->dpar.wmax + K.wpb - 1) / K.wpb;
    const int grid = c->dpar.persist ? std::max(1, std::min(need, sm * 16)) : need;
    k_dmc_move<T, NORD, MD><<<dim3(grid), block, K.smem, c->stream>>>(s, st, K.lay, c->dpar, c->dA,
                                                                     a.phase < 0 ? 0 : a.phase);
    break;
  }
  case Op::Tmove: {
    const int wl = a.dmc ? c->dpar.wmax : st.W;
    k_dmc_tmove<T, NORD, MD><<<dim3((wl + K.wpb - 1) / K.wpb), block, K.smem, c->stream>>>(
        s, st, K.lay, st.W, a.dmc ? c->dA.nw : nullptr, a.tau, a.variant, a.seed, a.dmc ? c->dA.ctr : nullptr,
        a.sweep0, a.moved);
    break;
  }
  case Op::DmcCopy: {
    k_dmc_copy<T><<<592, 128, 0, c->stream>>>(st, st2of<T>(c), c->dA, c->dB, c->N, c->C, c->dpar.wmax);
    break;
  }
  case Op::Vmc: {
    if (a.phase == 3 && c->el_staged && std::is_same<T, double>::value && !a.st_override) {
      // the E_L half of a sweep whose moves ran as phase 1
      ElRot rot{};
      rot.random = 1;
      rot.seed = a.seed;
      rot.sweep = a.sweep0;
      return run_el_staged<T, NORD, MD>(c, st, false, true, rot);
    }
    if (a.phase >= 0) {
      const bool acc6 = c->mover.kind == 6;
      auto kern = a.phase == 1 ? (acc6 ? k_vmc<T, NORD, MD, 1, 6> : k_vmc<T, NORD, MD, 1>)
                : a.phase == 2 ? k_vmc<T, NORD, MD, 2>
                : a.phase == 3 ? k_vmc<T, NORD, MD, 3> : (acc6 ? k_vmc<T, NORD, MD, 0, 6> : k_vmc<T, NORD, MD, 0>);
      // the accelerated mover of a mixed context takes the drift at the current position from the
      // FP64 state's orbital rows while they are current, and keeps them current
      const bool cache = std::is_same<T, float>::value && a.phase == 1 && acc6 && c->mover_cache && c->orb5_valid &&
                         c->prec == CHAMP_PREC_MIXED && !c->md.multidet && c->el_staged;
      if (!cache) c->orb5_valid = false;
      if (cache) {
        State<T> sc = st;
        sc.orb_cache = c->std_.orb5;
        kern<<<grid, block, K.smem, c->stream>>>(s, sc, K.lay, a.nsweep, a.seed, a.sweep0, a.step, c->reinv_every,
                                                 c->mover);
        break;
      }
      if (std::is_same<T, float>::value && a.phase == 1 && !acc6 && c->move_coop && c->kfm.lay.coop) {
        // the block's warps share the proposals' coefficient stream (move-only layout)
        const KCfg &M = c->kfm;
        kern<<<dim3((st.W + M.wpb - 1) / M.wpb), dim3(32 * M.wpb), M.smem, c->stream>>>(
            s, st, M.lay, a.nsweep, a.seed, a.sweep0, a.step, c->reinv_every, c->mover);
        break;
      }
      kern<<<grid, block, K.smem, c->stream>>>(s, st, K.lay, a.nsweep, a.seed, a.sweep0, a.step, c->reinv_every, c->mover);
      break;
    }
    CK(cudaMemsetAsync(st.s_esum, 0, sizeof(double) * st.W, c->stream));
    CK(cudaMemsetAsync(st.s_e2sum, 0, sizeof(double) * st.W, c->stream));
    CK(cudaMemsetAsync(st.s_acc, 0, sizeof(double) * st.W, c->stream));
    const bool tc = c->tc_on && !a.st_override;  // only FP32 contexts turn it on
    if (!tc) {
      auto kern = c->mover.kind == 6 ? k_vmc<T, NORD, MD, 0, 6> : k_vmc<T, NORD, MD, 0>;
      kern<<<grid, block, K.smem, c->stream>>>(s, st, K.lay, a.nsweep, a.seed, a.sweep0, a.step, c->reinv_every,
                                               c->mover);
      break;
    }
    // per sweep: moves, orbitals of all walkers on the tensor cores, E_L
    for (int isw = 0; isw < a.nsweep; isw++) {
      auto kmv = c->mover.kind == 6 ? k_vmc<T, NORD, MD, 1, 6> : k_vmc<T, NORD, MD, 1>;
      kmv<<<grid, block, K.smem, c->stream>>>(s, st, K.lay, 1, a.seed, a.sweep0 + isw, a.step, c->reinv_every,
                                              c->mover);
      CK(cudaGetLastError());
      int rc = run_orb_tc<T>(c, st);
      if (rc) return rc;
      k_vmc<T, NORD, MD, 2><<<grid, block, K.smem, c->stream>>>(s, st, K.lay, 1, a.seed, a.sweep0 + isw, a.step,
                                                                  c->reinv_every, c->mover);
      CK(cudaGetLastError());
    }
    break;
  }
  }
  CK(cudaGetLastError());
  return CHAMP_OK;
}

// One translation unit per (compute type, e-e-n order) instantiates its kernels through this macro
// (CHAMP_INST(f32, float, 4) defines launch_f32_n4 and attrs_f32_n4); launch_f32 / launch_f64
// dispatch on the context's e-e-n order.
#define CHAMP_INST(TAG, T, NORD)                                                                  \
  int launch_##TAG##_n##NORD(champ_ctx *c, Op op, const OpArgs &a) {                              \
    return c->md.multidet ? launch_t<T, NORD, true>(c, op, a) : launch_t<T, NORD, false>(c, op, a); \
  }                                                                                               \
  int attrs_##TAG##_n##NORD(champ_ctx *c) {                                                       \
    return c->md.multidet ? set_smem_attrs<T, NORD, true>(c) : set_smem_attrs<T, NORD, false>(c); \
  }

#undef fail
