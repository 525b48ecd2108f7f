// ctx.h -- host-side context of the engine, shared by the C-ABI translation unit and
// the per-precision kernel instantiation units.
#pragma once
#include <string>
#include <vector>

#include "kernels.cuh"

int champ_fail(int code, const std::string &msg);
#define CK(call)                                                                                          \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess) return champ_fail(CHAMP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Occupied orbitals and determinant tables of the wave function (occ_bld, excit_bld,
// cdet_in_wf_bld: deriv_fast_mod.f90:144-300), built once on the host.
struct MultiDet {
  int multidet = 0, ndet = 0;
  int nocc[2] = {0, 0}, nvirt[2] = {0, 0}, ndu[2] = {0, 0};
  std::vector<int> occ[2];              // orbital index of each occupied column
  std::vector<int> dk[2], dh[2], dp[2];  // per unique determinant: order, holes[4], particles[4]
  std::vector<double> dsg[2];
  std::vector<int> ciu, cid;
  std::vector<double> ccoef;
};

// The optimisable parameters in the caller's layouts (champ_system), kept for champ_set_params /
// champ_apply_param_step, and the structure needed to re-derive what the kernels use.
struct Params {
  std::vector<double> a4, b, c, csf, coef;  // [nct][norda+1], [nspin2b][nordb+1], [nct][nterms] as given,
                                            // [ncsf], [norb][nbasis] (input basis order)
  std::vector<int> csf_ndet, csf_det;
  std::vector<double> csf_det_coef;
  int norda = 0, nordb = 0, nordc = 0, nspin2b = 1, een_cusp = 0, nterms = 0;
  double scalek = 1;
  std::vector<int> cfree;  // free e-e-n coefficients of a centre type (term indices)
};

// Largest per-warp shared-memory footprint for which a walker's state stays resident in
// shared memory inside the fused kernels (keeps >= 16 warps per SM).
constexpr size_t RESIDENT_LIMIT = 12 * 1024;

// Launch configuration of the kernels of one compute type: per-warp shared-memory layout,
// dynamic shared memory per block and warps (walkers) per block.
struct KCfg {
  Layout lay{};
  size_t smem = 0;
  int wpb = 4;
};

struct champ_ctx {
  int prec = 0;
  cudaStream_t stream = nullptr;
  int wmax = 0, W = 0;
  int N = 0, nup = 0, ndn = 0, C = 0, nct = 0, nshell = 0, nbasis = 0, nmax = 0, nordc = 0, nloc = 0;
  int nomax = 1;
  MultiDet md;
  Params par;
  std::vector<int> perm_b;  // internal basis index -> caller's basis index
  // numerical radial tables (kind-2 shells), prepared at create: per table (grid, points, first
  // value index, 0), 10 parameters (r0, h, log h, c0..c4, a0, ak), values and spline second
  // derivatives of all tables one after another; shell -> table
  std::vector<int4> rad_tab;
  std::vector<double> rad_par, rad_y, rad_y2;
  std::vector<int> rad_shell;
  // opt-in device timing of the VMC sweep kernels (option "phase_timing"): event pairs per
  // launch, summed per phase by champ_phase_times
  int ptime = 0;
  std::vector<void *> ev_pool;             // cudaEvent_t, reused
  std::vector<std::pair<int, int>> ev_use; // (phase, index of the start event; stop = index + 1)
  std::vector<void *> allocs;
  Sys<double> sd;
  Sys<float> sf;
  State<double> std_;
  State<float> stf;
  double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  bool have_walkers = false;
  KCfg kf, kd;  // FP32 and FP64 kernels (a mixed-precision context uses both)
  KCfg kfm;     // FP32 Gaussian moves of a state in HBM sharing the coefficient stream (kfm.lay.coop)
  int move_coop = 0;  // option "move_coop": 1 runs those moves with kfm
  int orb_coop_ok = 0, orb_coop = 0;  // k_el_orb's warps share the coefficient stream (option "orb_coop")
  size_t orb_stage = 0;               // offset of its double buffer in the block's shared memory
  bool orb5_valid = false;  // the FP64 state's orbital rows are current for the walkers' positions
  int mover_cache = 1;      // option "mover_cache": the accelerated mover's drift from those rows
  // staged evaluation (elstage.cuh) of the FP64 state when it lives in HBM: on/off (option
  // "staged_eval"), warps per block and dynamic shared memory of k_el_jas, k_el_orb, k_el_fin,
  // and the pseudopotential scratch of k_el_fin (elements)
  // the VMC mover (champ_set_mover): Gaussian displacements, or the accelerated Metropolis method
  Mover mover{1, 5.0, 1.0, 1.0};
  int el_staged = 0;
  int el_wpb[3] = {4, 4, 4};
  size_t el_smem[3] = {0, 0, 0};
  int el_nscr = 0;
  // device staging for per-call host arrays
  double *d_in = nullptr, *d_out = nullptr;
  uint8_t *d_mask = nullptr;
  int nparm_jas = 0;
  // parameter derivatives and O/H accumulation
  int np_raw = 0;          // raw Jastrow parameters on the device (a, b, all c terms)
  int ncfree = 0;          // free e-e-n coefficients per centre type
  int ncsfp = 0, norbp = 0;  // CSF and orbital-rotation parameters
  int norb = 0;
  double *call_d = nullptr;  // [nbasis][norb] coefficients of all orbitals in FP64 (B-matrix GEMM)
  std::vector<int4> orbp;  // (i, j, antisymmetric, 0)
  double *pg_scr = nullptr;
  size_t scr_stride = 0;
  std::vector<double> cproj;
  int nfree = 0;           // free parameters reported
  size_t smem_pg = 0;      // dynamic shared memory of the derivative kernel
  int wpb_pg = 4;
  int pg_lanesum = 0;      // per-lane slots for the NLPP parameter sums in the derivative kernel
  double *pg_dl = nullptr, *pg_de = nullptr, *pg_el = nullptr, *pg_wt = nullptr;
  // tape of the parameter-gradient forward pass (see PGOut)
  double *pg_tv = nullptr, *pg_tc = nullptr;
  int *pg_tn = nullptr;
  bool have_tape = false;
  int pg_mode = 0;  // 0: forward pass + reverse sweep; 1: one fused pass
  int nquad = 12;   // points of the nonlocal quadrature rule in use
  QuadRule quad{};  // its points and weights (host copy)
  double *oh_oa = nullptr, *oh_ow = nullptr, *oh_mb = nullptr, *oh_s = nullptr, *oh_h = nullptr;
  bool have_pgrad = false;
  void *cublas = nullptr;
  // DMC: second state buffer for branching, per-walker weights/energies, device scalars
  bool dmc_ready = false;
  DmcPar dpar{};
  DmcData dA, dB;
  State<double> std2;
  State<float> stf2;
  void *scan_tmp = nullptr;
  size_t scan_bytes = 0;
  int dmc_step = 0;
  // CUDA graph of two DMC steps (A->B->A buffers), captured on a private stream, replayed per pair
  int dmc_graph_on = 1;
  int dmc_ene_int = 1;  // DMC energy integration over the step: 1 ene_int_v9, 0 none (option "dmc_ene_int")
  void *dmc_graph = nullptr, *dmc_exec = nullptr;  // cudaGraph_t, cudaGraphExec_t
  uint64_t dmc_graph_seed = 0;
  cudaStream_t cap_stream = nullptr;
  // tensor-core orbital contraction of the full evaluation (mixed precision, state in HBM)
  int num_sms = 0;
  int reinv_every = 1;            // VMC sweeps between FP64 re-inversions of the Slater matrices
  int tc_on = 0, tc_ok = 0;       // in use; supported for this system and precision
  int tc_Kp = 0, tc_Np[2] = {0, 0}, tc_ncols[2] = {32, 32};
  float *tc_phi = nullptr;        // [wmax*N*5][Kp] basis rows
  float *tc_b[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [spin][hi, lo]: [Np][Kp]
  int *tc_err = nullptr;          // set by a contraction that gave up waiting
  std::vector<float> tc_coef[2];  // host copy of the occupied coefficients [nbasis][nocc]
  std::vector<int> tc_shl;        // host copy of the shells' l (internal basis order)
  // fused basis + contraction (orbfused.cuh): padded K layout and split coefficients
  int tc_fused_ok = 0, tc_mode = 0;  // fused kernel supported; mode in use: 1 fused, 2 basis rows + product
  int tc_kchunk = 4;                 // fused kernel: K-blocks per TMEM accumulation chunk (0: all)
  int tc_kq = 0, tc_nkb = 0, tc_fcols[2] = {32, 32};
  std::vector<int> tc_kpos_h, tc_b0_h;  // host copies: padded position and first basis function per shell
  int *tc_blk_sh = nullptr, *tc_kpos = nullptr;
  float *tc_bf[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [spin][hi, lo]: [Np][Kq]
};

template <class T>
inline Sys<T> &sysof(champ_ctx *c);
template <>
inline Sys<double> &sysof<double>(champ_ctx *c) { return c->sd; }
template <>
inline Sys<float> &sysof<float>(champ_ctx *c) { return c->sf; }
template <class T>
inline State<T> &stof(champ_ctx *c);
template <>
inline State<double> &stof<double>(champ_ctx *c) { return c->std_; }
template <>
inline State<float> &stof<float>(champ_ctx *c) { return c->stf; }

template <class T>
inline State<T> &st2of(champ_ctx *c);
template <>
inline State<double> &st2of<double>(champ_ctx *c) { return c->std2; }
template <>
inline State<float> &st2of<float>(champ_ctx *c) { return c->stf2; }

template <class T>
inline KCfg &kcfg(champ_ctx *c);
template <>
inline KCfg &kcfg<double>(champ_ctx *c) { return c->kd; }
template <>
inline KCfg &kcfg<float>(champ_ctx *c) { return c->kf; }

enum class Op { Eval, EvalOut, Propose, ProposeGrad, Accept, Vmc, PGrad, PGradBwd, DmcMove, DmcCopy, Tmove };
struct OpArgs {
  int e = 0;
  const double *xnew = nullptr;
  double *ratio = nullptr, *grad = nullptr;
  const uint8_t *mask = nullptr;
  int nsweep = 0;
  uint64_t seed = 0, sweep0 = 0;
  double step = 0;
  PGOut pgout;
  int istep = 0;
  const void *st_override = nullptr;  // State<T> to use instead of the context's (and its walker count)
  int nw_override = 0;
  int phase = -1;  // Vmc: one k_vmc launch of this phase (no statistics reset); DmcMove: k_dmc_move phase
  bool rebuild = false;  // Eval: only the state the moves need (inverse, log-det, move tables), no E_L
  // Tmove: time step, variant (1 casula1, 2 det_balance1), per-walker counts of accepted T-moves
  // (device, may be null), and whether the walker count and step number come from the DMC state
  double tau = 0;
  int variant = 0;
  int *moved = nullptr;
  bool dmc = false;
};


// kernel launchers per (compute type, e-e-n order), one translation unit each (inst_*.cu)
#define CHAMP_DECL(TAG, NORD)                                    \
  int launch_##TAG##_n##NORD(champ_ctx *c, Op op, const OpArgs &a); \
  int attrs_##TAG##_n##NORD(champ_ctx *c);
CHAMP_DECL(f32, 0) CHAMP_DECL(f32, 4) CHAMP_DECL(f32, 5)
CHAMP_DECL(f64, 0) CHAMP_DECL(f64, 4) CHAMP_DECL(f64, 5)
#undef CHAMP_DECL

int champ_fail(int code, const std::string &msg);
inline int launch_f32(champ_ctx *c, Op op, const OpArgs &a) {
  switch (c->nordc) {
  case 0: case 1: return launch_f32_n0(c, op, a);
  case 4: return launch_f32_n4(c, op, a);
  case 5: return launch_f32_n5(c, op, a);
  default: return champ_fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
inline int launch_f64(champ_ctx *c, Op op, const OpArgs &a) {
  switch (c->nordc) {
  case 0: case 1: return launch_f64_n0(c, op, a);
  case 4: return launch_f64_n4(c, op, a);
  case 5: return launch_f64_n5(c, op, a);
  default: return champ_fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
inline int attrs_f32(champ_ctx *c) {
  switch (c->nordc) {
  case 0: case 1: return attrs_f32_n0(c);
  case 4: return attrs_f32_n4(c);
  case 5: return attrs_f32_n5(c);
  default: return champ_fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
inline int attrs_f64(champ_ctx *c) {
  switch (c->nordc) {
  case 0: case 1: return attrs_f64_n0(c);
  case 4: return attrs_f64_n4(c);
  case 5: return attrs_f64_n5(c);
  default: return champ_fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
