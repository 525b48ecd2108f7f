/*
 * champ_b200.h -- C ABI of the walker-batched Slater-Jastrow engine.
 *
 * The engine evaluates, for all walkers at once on one B200, what CHAMP's
 * per-walker wave-function routines evaluate one walker at a time:
 *
 *   champ_eval_full   <->  hpsi            (qmc/vmc/hpsi.f90:2)
 *   champ_propose_1e  <->  hpsie           (qmc/vmc/hpsie.f90:1)
 *   champ_accept_1e   <->  jassav + detsav + dete_save
 *                          (qmc/vmc/jassav.f90:1, qmc/vmc/detsav.f90:1, qmc/dete_mod.f90:75)
 *   champ_grad_1e     <->  eval_grad / calc_1e_derivatives
 *                          (qmc/dete_mod.f90:249, qmc/psi_utils_mod.f90:457)
 *   champ_set_walkers <->  psi_at for every walker (qmc/psi_utils_mod.f90:13)
 *   champ_vmc_sweeps  <->  the metrop_mov1 sweep loop + hpsi per sweep
 *                          (qmc/vmc/metrop_mov1.f90:64-296, qmc/vmc/vmc.f90:250-331)
 *   champ_dmc_init/champ_dmc_steps <-> rundmc walker/electron loops, split_join
 *                          (qmc/rundmc_mod.f90:123-365)
 *   champ_param_grad  <->  dpsi_bld / deloc_bld (qmc/deriv_mod.f90:248,437)
 *   champ_accumulate_oh <-> dpsi_dpsi / dpsi_deloc / dpsi_dpsi_eloc averages
 *                          (qmc/deriv_mod.f90:683,1375,898)
 *
 * Conventions
 *   - All indices are 0-based.  Electrons 0..nup-1 are spin up, nup..nelec-1 spin down.
 *   - Host arrays are C row-major.  Walker arrays are walker-major: x[w][e][k].
 *   - Every entry point returns 0 on success and a positive CHAMP_E* code on error;
 *     champ_last_error() gives a message.  Nothing calls exit() or traps.
 *   - A context owns its device buffers and works on the CUDA stream given at create.
 */
#ifndef CHAMP_B200_H
#define CHAMP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAMP_OK 0
#define CHAMP_EINVAL 1      /* bad argument or size beyond the compiled limits */
#define CHAMP_ECUDA 2       /* CUDA runtime error */
#define CHAMP_ENOMEM 3      /* device allocation failed */
#define CHAMP_ESTATE 4      /* call out of order (e.g. propose before set_walkers) */
#define CHAMP_ESINGULAR 5   /* a walker hit a singular Slater matrix (see champ_walker_status) */

#define CHAMP_PREC_FP64 0   /* every step in FP64 */
#define CHAMP_PREC_MIXED 1  /* single-electron moves (basis and orbitals at the proposed position,
                               Jastrow pair values, ratio and drift) in FP32 with FP32 Jastrow and
                               distance tables; the accepted Sherman-Morrison update, the inverse
                               and log-det in FP64; every full evaluation (E_L, velocities, the
                               nonlocal quadrature, parameter derivatives) in FP64 from the
                               positions, re-inverting the Slater matrices and refreshing the FP32
                               tables.  E_L therefore equals the FP64 engine's on the same
                               configuration; FP32 only steers the Metropolis acceptance. */
#define CHAMP_PREC_FP32 2   /* as MIXED, but the full evaluation also in FP32 (orbitals optionally
                               on the tensor cores, option "orbital_tc"): inverse, log-det, the
                               Sherman-Morrison update and the E_L sums stay FP64.  E_L carries
                               FP32-level relative errors (1e-7 of |lap ln psi|), which exceed
                               1e-6 Ha on systems with large kinetic energies. */

/* Per-walker status bits (champ_walker_status). */
#define CHAMP_WS_SINGULAR 1u   /* Slater matrix singular at the last full evaluation */
#define CHAMP_WS_NONFINITE 2u  /* non-finite E_L or ln|psi| */

/* Maximum sizes the kernels are compiled for. */
#define CHAMP_MAX_ELEC 256
#define CHAMP_MAX_SPIN 64      /* electrons of one spin */
#define CHAMP_MAX_L 4
#define CHAMP_MAX_CTYPE 4      /* nuclear (centre) types */
#define CHAMP_MAX_NORD 7
#define CHAMP_MAX_LCHAN 5      /* pseudopotential l channels (npotd) */
#define CHAMP_MAX_QUAD 86      /* nonlocal quadrature points */

/*
 * System descriptor: everything the reference reads from its input menus
 * (nuclei, basis, orbitals, csfs, jastrow, pseudo blocks).  Pointers are host
 * pointers; they are copied at champ_create and may be freed afterwards.
 */
typedef struct champ_system {
  int32_t nelec, nup;
  int32_t ncent, nctype;
  const double *cent;          /* [ncent][3] */
  const int32_t *iwctype;      /* [ncent] centre type */
  const double *znuc;          /* [nctype] nuclear (or pseudo-atom) charge */

  /* Basis (qmc/vmc/basis_fns.f90:38-474): a shell is one radial function on one centre,
     R(r) = sum_p coef_p * N(n,l,zeta_p) * r^(n-1) * exp(-zeta_p r)     (Slater, kind 0)
                                          * exp(-zeta_p r^2)   (Gaussian, kind 1)
     R(r) = coef_0 * sqrt((2l+1)/4pi) * f(r)    (numerical, kind 2: f is radial table
                                                 shell_rad[ish], one primitive)
     N is the reference normalisation (qmc/vmc/basis_norm.f90), including sqrt((2l+1)/4pi).
     Basis function b = R_shell(b)(r) * C_{l,m}(rhat), C the real harmonics of basis_fns. */
  int32_t nshell;
  const int32_t *shell_cent;   /* [nshell] */
  const int32_t *shell_n;      /* [nshell] */
  const int32_t *shell_l;      /* [nshell] 0..4 */
  const int32_t *shell_kind;   /* [nshell] 0 Slater, 1 Gaussian, 2 numerical radial table */
  const int32_t *shell_nprim;  /* [nshell] */
  const double *prim_zeta;     /* [sum nprim] */
  const double *prim_coef;     /* [sum nprim] contraction weights */
  int32_t nbasis;
  const int32_t *basis_shell;  /* [nbasis] shell of basis function; shells contiguous */
  const int32_t *basis_m;      /* [nbasis] m in -l..l (x=+1, y=-1, z=0 for l=1) */

  /* Orbitals: orb_i = sum_b coef[i][b] * basis_b  (coef(ibasis,iorb) in the reference). */
  int32_t norb;
  const double *coef;          /* [norb][nbasis] */

  /* Determinants and CSFs (qmc/csfs_mod.f90, qmc/deriv_fast_mod.f90:144). */
  int32_t ndet;
  const int32_t *det_orb;      /* [ndet][nelec] orbital in column j (iworbd) */
  int32_t ncsf;
  const double *csf_coef;      /* [ncsf] */
  const int32_t *csf_ndet;     /* [ncsf] */
  const int32_t *csf_det;      /* [sum csf_ndet] determinant index */
  const double *csf_det_coef;  /* [sum csf_ndet] (cdet_in_csf) */

  /* Jastrow ijas=4, isc=4 (qmc/vmc/jastrow4.f90, qmc/vmc/scale_dist.f90). */
  double scalek;
  int32_t norda, nordb, nordc;
  int32_t nspin2b;             /* 1: one b set (parallel spins get 1/2 on b1); 2: separate sets */
  int32_t een_cusp;            /* nonzero: dependent e-e-n coefficients are set from the
                                  cusp conditions (qmc/fit/cuspinit4.f90, cuspexact4.f90) */
  const double *a4;            /* [nctype][norda+1] */
  const double *b;             /* [nspin2b][nordb+1] */
  const double *c;             /* [nctype][nterms4(nordc)] */

  /* Pseudopotential (nloc=6: Gaussian ECP, qmc/vmc/readps_gauss.f90:126-165). */
  int32_t nloc;                /* 0 all-electron, 6 Gaussian ECP */
  int32_t nquad;               /* quadrature points of the nonlocal integration: the rule of
                                  qmc/vmc/rotqua.f90 (gesqua) with the number of points closest
                                  to nquad among 4, 6, 12, 18, 20, 24, 26, 32, 50, 86 */
  int32_t mgauss;              /* max terms per channel */
  const int32_t *npotd;        /* [nctype] number of l channels */
  const int32_t *lpotp1;       /* [nctype] 1-based local channel */
  const int32_t *necp_term;    /* [nctype][CHAMP_MAX_LCHAN] terms of channel l (0-based l) */
  const int32_t *necp_power;   /* [nctype][CHAMP_MAX_LCHAN][mgauss] */
  const double *ecp_coef;      /* [nctype][CHAMP_MAX_LCHAN][mgauss] */
  const double *ecp_exponent;  /* [nctype][CHAMP_MAX_LCHAN][mgauss] */

  /* Numerical radial functions (numr=1: the basis.<centre type> grids of read_bas_num.f90,
     interpolated as splfit_bas does, qmc/vmc/splfit.f90): a cubic spline through the grid values
     with end slopes from a 5-point polynomial fit at small r and an exponential a0 exp(-ak r)
     matched at the last point, which also continues the function beyond the grid. */
  int32_t nrad;                /* radial tables (0: none) */
  const int32_t *rad_igrid;    /* [nrad] grid: 1 linear r(i) = r0 + (i-1) h; 2 exponential
                                  r(i) = r0 h^(i-1); 3 shifted exponential r(i) = r0 (h^(i-1) - 1) */
  const int32_t *rad_nr;       /* [nrad] grid points (>= 6) */
  const double *rad_h;         /* [nrad] exp_h_bas: the step (grid 1) or the ratio (grids 2, 3) */
  const double *rad_r0;        /* [nrad] r0_bas as read: first point (grids 1, 2) or last point (3) */
  const double *rad_x;         /* [sum rad_nr] grid points, tables one after another */
  const double *rad_val;       /* [sum rad_nr] function values at the grid points */
  const int32_t *shell_rad;    /* [nshell] radial table of each kind-2 shell (others ignored) */
} champ_system;

/* Outputs of a full evaluation (hpsi).  Host pointers; any may be NULL. */
typedef struct champ_eval_out {
  double *lnpsi;     /* [nw] ln|psi| = ln|D| + J */
  double *sign;      /* [nw] sign of D */
  double *psij;      /* [nw] J = ln(Jastrow) */
  double *velocity;  /* [nw][nelec][3] grad ln psi */
  double *div_v;     /* [nw][nelec] */
  double *d2lnpsi;   /* [nw] sum_i lap_i ln psi */
  double *pe;        /* [nw] total potential energy (local + nonlocal + e-e + n-n) */
  double *pe_ee;     /* [nw] e-e Coulomb energy (pei) */
  double *pe_nonloc; /* [nw] nonlocal pseudopotential energy */
  double *energy;    /* [nw] local energy E_L */
} champ_eval_out;

/* Per-walker VMC accumulators (acues1 in the reference).  Host pointers; any may be NULL. */
typedef struct champ_vmc_stats {
  double *esum;      /* [nw] sum of E_L over the sweeps of the call */
  double *e2sum;     /* [nw] sum of E_L^2 */
  double *accept;    /* [nw] accepted single-electron moves */
  double *elast;     /* [nw] E_L after the last sweep */
} champ_vmc_stats;

typedef struct champ_ctx champ_ctx;

const char *champ_last_error(void);
const char *champ_version(void);

/* Context. precision = CHAMP_PREC_*; stream = cudaStream_t (NULL: default stream). */
int champ_create(const champ_system *sys, int32_t w_max, int32_t precision, void *stream,
                 champ_ctx **out);
int champ_destroy(champ_ctx *ctx);
int champ_nparam(const champ_ctx *ctx, int32_t *nparm_jas, int32_t *nparm_csf, int32_t *nparm_orb);

/* Walker positions.  psi_at for every walker: sets x and runs a full evaluation,
   rebuilding inverses and Jastrow tables (qmc/psi_utils_mod.f90:13). */
int champ_set_walkers(champ_ctx *ctx, int32_t nw, const double *x /* host [nw][nelec][3] */);
int champ_get_walkers(champ_ctx *ctx, double *x /* host [nw][nelec][3] */);

/* Rotation applied to the nonlocal quadrature grid (rotqua, qmc/vmc/rotqua.f90:621).
   rot = row-major 3x3 orthogonal matrix; NULL resets to the identity. */
int champ_set_quadrature_rotation(champ_ctx *ctx, const double *rot);

/* hpsi for all walkers at their current positions. */
int champ_eval_full(champ_ctx *ctx, const champ_eval_out *out);

/* hpsie: psi(x with electron iel at xnew)/psi(x) for every walker, and grad ln psi of
   electron iel at the new position (grad_new may be NULL). */
int champ_propose_1e(champ_ctx *ctx, int32_t iel, const double *xnew /* [nw][3] */,
                     double *ratio /* [nw] */, double *grad_new /* [nw][3] or NULL */);
/* Accept the last proposal of electron iel where accept[w] != 0. */
int champ_accept_1e(champ_ctx *ctx, int32_t iel, const uint8_t *accept /* [nw] */);
/* grad ln psi of electron iel at the current positions. */
int champ_grad_1e(champ_ctx *ctx, int32_t iel, double *grad /* [nw][3] */);

/* Fused VMC: nsweep sweeps of single-electron Metropolis moves (Gaussian proposal of
   width step), with a full E_L evaluation after every sweep, all on the device.
   Random numbers come from a counter-based generator keyed by (seed, walker, sweep). */
int champ_vmc_sweeps(champ_ctx *ctx, int32_t nsweep, uint64_t seed, uint64_t sweep0,
                     double step, const champ_vmc_stats *stats);

/* Same as champ_vmc_sweeps, but the walkers come from and go back to host memory and
   the per-walker E_L of the last sweep is copied back (the call a host driver makes).  The state
   the moves start from (inverses, log-determinants, move tables) is rebuilt from the incoming
   positions without an E_L evaluation of them. */
int champ_vmc_run_host(champ_ctx *ctx, int32_t nw, double *x /* host [nw][nelec][3], in/out */,
                       int32_t nsweep, uint64_t seed, uint64_t sweep0, double step,
                       double *eloc /* host [nw] */);

/* Parameter derivatives for the linear method (dpsi_bld / deloc_bld, qmc/deriv_mod.f90:248,437;
   Jastrow parts: deriv_jastrow4, qmc/vmc/deriv_jastrow4.f90, and deriv_nonloc_pot,
   qmc/fit/deriv_nonloc_pot.f90), for every walker at its current position: d ln psi / dp and
   dE_L / dp for the P = champ_nparam() free parameters, ordered as the reference orders them
   (Jastrow: a_3..a_{norda+1} per centre type, b_2..b_{nordb+1} per b set, then the free e-e-n
   coefficients per centre type, i.e. those the cusp conditions do not fix).  Host outputs may
   be NULL; the results stay on the device for champ_accumulate_oh. */
int champ_param_grad(champ_ctx *ctx, double *dlnpsi /* [nw][P] */, double *deloc /* [nw][P] */,
                     double *eloc /* [nw] */);
/* The same derivatives as a forward / backward pair (the reference's forward derivative chains,
   qmc/vmc/deriv_jastrow4.f90, qmc/fit/deriv_nonloc.f90, qmc/deriv_orb_mod.f90:1486,1557, and
   qmc/deriv_csf_mod.f90, replaced by one reverse sweep).  champ_param_grad_fwd evaluates E_L
   (FP64 in FP64 and mixed precision) and keeps on the device a tape: each walker's velocities,
   the coefficients of its nonlocal quadrature points and the orbital-resolved local energy.
   champ_param_grad_bwd sweeps once in reverse: with the adjoint seeds -1/2 on every electron's
   Laplacian of ln J, -grad ln psi on its gradient and each quadrature point's coefficient on
   the change of ln J when its electron moves there, it accumulates d ln psi/dp and dE_L/dp for
   all Jastrow parameters from the pair, e-n and point terms recomputed from the positions
   (in FP32 for mixed precision, FP64 otherwise), then contracts the orbital-resolved local
   energy for the CSF and orbital-rotation parameters (FP64).  champ_param_grad runs both (or,
   with option "param_grad_mode" 1, one fused FP64/FP32 pass).  Outputs as champ_param_grad;
   the bwd call consumes the tape (CHAMP_ESTATE without a preceding fwd). */
int champ_param_grad_fwd(champ_ctx *ctx, double *eloc /* [nw] or NULL */);
int champ_param_grad_bwd(champ_ctx *ctx, double *dlnpsi /* [nw][P] or NULL */, double *deloc /* [nw][P] or NULL */);
/* O/H accumulation of the linear method (dpsi_dpsi / dpsi_deloc / dpsi_dpsi_eloc averages,
   qmc/deriv_mod.f90:683,898,1375; opt_lin_mod.f90:249,404) over the walkers of the last
   champ_param_grad, with optional weights: with Oa = (1, dlnpsi) and Mb = (E_L, E_L dlnpsi + deloc),
   S[a][b] = sum_w wt_w Oa_a Oa_b and H[a][b] = sum_w wt_w Oa_a Mb_b, row-major (P+1)x(P+1), in FP64. */
int champ_accumulate_oh(champ_ctx *ctx, const double *weights /* [nw] or NULL */, double *S, double *H);
/* Device addresses of the O/H accumulators that champ_accumulate_oh fills (row-major
   (P+1)x(P+1) FP64, owned by the context, valid until champ_destroy), for a caller that reduces
   them across ranks on the device (the MPI reduction of the averages in the reference,
   deriv_mod.f90:683,898,1375) without copying them to the host. */
int champ_oh_buffers(const champ_ctx *ctx, const double **S, const double **H);

/* Wave-function parameters of a live context (no counterpart as one call in the reference, whose
   optimiser writes the new parameters into its global arrays; the layouts are champ_system's):
   a4 [nctype][norda+1], b [nspin2b][nordb+1], c [nctype][nterms4(nordc)], csf_coef [ncsf],
   coef [norb][nbasis].  NULL arrays are left as they are.  The e-e-n coefficients the cusp
   conditions fix are re-derived from the others (champ_get_params returns them derived).  The
   current walkers are re-evaluated for the new wave function (as champ_set_walkers does); the
   tape of champ_param_grad_fwd and the results of champ_param_grad are invalidated. */
int champ_set_params(champ_ctx *ctx, const double *a4, const double *b, const double *c, const double *csf_coef,
                     const double *coef);
int champ_get_params(const champ_ctx *ctx, double *a4, double *b, double *c, double *csf_coef, double *coef);
/* Adds a step dp[P] in the order of champ_param_grad's parameters (CSF coefficients 2..ncsf,
   orbital rotations: coefficients of orbital i += dp times those of orbital j, and those of j -=
   dp times those of i for a rotation between two active orbitals, then the free Jastrow
   parameters) -- the update the linear method's delta_lin makes -- and re-evaluates the walkers. */
int champ_apply_param_step(champ_ctx *ctx, const double *dp /* [P] */);

/* Linear-method update (ovlp_lin_bld, ham_lin_energy_bld, ham_lin_renorm_stab_bld and
   delta_lin_bld, qmc/opt_lin_mod.f90:249-1265; host code, no context or GPU needed).  S and H are
   the (nparm+1)^2 sums of champ_accumulate_oh (possibly summed over ranks); the first ncsf
   parameters are CSF coefficients (the engine's parameter order puts them first).  Builds the
   overlap and Hamiltonian of the wave function and its derivatives, renormalises them by the
   overlap's diagonal, adds diag_stab to the Hamiltonian's diagonal (stabilization 'identity'),
   solves H c = E S c, and selects the eigenvector as the reference does by default: the lowest
   eigenvalue inside (E - sigma, E + 0.01) (E = the current energy, sigma its standard deviation;
   sigma <= 0: no lower bound) unless its wave-function variation exceeds 100 times the smallest
   one, else the one with the smallest variation (select 0; 1: lowest in the window, 2: largest
   first component, 3: smallest variation).  dp[nparm] receives the parameter variations with the
   semi-orthogonal normalisation (update_nonlinear 'semiorthogonal', xi = 1); parameters with no
   variance get 0.  info (may be NULL): [selected eigenvalue, lowest eigenvalue, wave-function
   variation of the selection, parameters kept]. */
int champ_linear_update(int32_t nparm, int32_t ncsf, const double *S, const double *H, double sigma,
                        double diag_stab, int32_t select, double *dp, double *info /* [4] or NULL */);

/* The checks the reference's optimisation driver makes on a step before it keeps it
   (wf_update_and_check, qmc/optimization_mod.f90:1730-1840): *bad = 1 if the root-mean-square
   variation of the CSF coefficients exceeds 1, of the Jastrow parameters max(10, 5/scalek), of all
   parameters 10 (each over the parameters the step changes), or psi_lin_var_norm (info[2] of
   champ_linear_update) exceeds 10, or b2 (a2) would exceed 100; *bad = 2 if b2 or a2 would fall
   below -scalek (a pole of the Pade form) or dp is not finite; else 0. */
int champ_check_param_step(const champ_ctx *ctx, const double *dp /* [P] */, double psi_lin_var_norm, int32_t *bad);

/* Correlated sampling of a trial step on the current walkers: E_L of every walker for the
   parameters + dp, and ln|psi_new| - ln|psi_old| (the walkers' reweighting is exp(2 dlnpsi)).
   The context's parameters and walker state are unchanged afterwards. */
int champ_eval_param_step(champ_ctx *ctx, const double *dp /* [P] */, double *eloc /* [nw] or NULL */,
                          double *dlnpsi /* [nw] or NULL */);

/* One linear-method iteration with the reference's stabilisation search (adjust_diag_stab and
   wf_update_and_check_and_stab, qmc/optimization_mod.f90:1845-2250; quad_min.f90): steps for
   add_diag, add_diag/10 and 10 add_diag (*diag_stab = add_diag on input) from the sums S, H over
   the parameters sel[nsel] (increasing indices; sel NULL: all P parameters); bad steps multiply
   add_diag by 10^(sum of the bad codes, at most 3); the three trial wave functions' energies by
   correlated sampling on the current walkers (reweighted; a trial whose weights' effective sample
   size falls below 1/50 of the walkers is not reliable); if all three are much worse than the
   current energy (sigma above (2.5 - p_var) times, or the energy above 3 (1 + p_var) combined
   errors) add_diag is multiplied by 1000; then the objective (1 - p_var) E + p_var sigma^2 fitted
   by a parabola in log10(add_diag) gives the final constant (bounded to two decades), which is
   raised by factors of 10 until the step passes champ_check_param_step.  Applies that step to the
   context and returns it in dp (host [P] or NULL), the final constant in *diag_stab and info
   (host [8] or NULL): [eigenvalue, wave-function variation, current energy, its error, correlated
   energies of the three trial constants, search iterations]. */
int champ_linear_method_step(champ_ctx *ctx, int32_t nsel, const int32_t *sel, const double *S, const double *H,
                             double sigma, double p_var, double *diag_stab, double *dp, double *info);

/* Diffusion Monte Carlo (rundmc, qmc/rundmc_mod.f90:17-422).  champ_dmc_init starts from the
   current walkers (weight 1); w_target is the target population and the trial energy follows
   E_T = E_g - ln(W / w_target) / (gpop * tau), E_g a running average of the growth energy
   E_T - ln(sum w_new / W) / tau, seeded with the median local energy.  The population may range
   up to w_max.
   champ_dmc_steps runs nstep steps (drift-diffusion moves with the Green's-function acceptance
   of green_functions_mod.f90, E_L, reweighting, branching) without host synchronisation and
   returns per step {population, sum w, sum w E_L, E_T} in stats (host [nstep][4] or NULL).
   Afterwards the context's walker count is the new population.  Pairs of steps run as one
   CUDA graph (captured on first use and whenever the seed changes; option "dmc_graph" 0 launches
   step by step); the step number that keys the random numbers is kept on the device.  The
   reweighting integrates the energy over the step as the reference's default ene_int_v9 does
   (green_functions_mod.f90:382-472, limit_rewt_dmc 10, c_rewt 3.5, effective time step of
   itau_eff 1); option "dmc_ene_int" 0 uses the plain local energies (no_ene_int). */
int champ_dmc_init(champ_ctx *ctx, int32_t w_target, double tau, double gpop);
int champ_dmc_steps(champ_ctx *ctx, int32_t nstep, uint64_t seed, double *stats);

int champ_walker_status(champ_ctx *ctx, uint32_t *flags /* [nw] */);
/* Current number of walkers (changes with DMC branching). */
int champ_num_walkers(const champ_ctx *ctx, int32_t *nw);

/* Local energy without allocation (no counterpart in the reference: an addition for callers
   that cannot allocate device memory, such as host codes whose GPU memory is wholly owned by
   their own pool allocator or that must not allocate inside a time-critical loop).
   x and eloc are DEVICE pointers the caller owns (x[nw][nelec][3], eloc[nw]); E_L is
   evaluated as champ_eval_full does, on the context's stream, with the quadrature rotation
   of champ_set_quadrature_rotation.  Intermediates live in one fixed 16 MiB device array
   compiled into the library: nw beyond what fits returns CHAMP_EINVAL with the limit in
   champ_last_error().  The first call on a device looks the array's address up.  The call
   makes no device allocation; it leaves the context's walkers untouched.  In FP32 precision it
   computes the orbitals on the CUDA cores (the tensor-core contraction of option "orbital_tc" is
   not used here); mixed precision evaluates in FP64 as champ_eval_full does.  All calls share the
   array, so calls that overlap on the GPU (other streams, other contexts on the device) race. */
int champ_eval_energy_noalloc(champ_ctx *ctx, int32_t nw, const double *x, double *eloc);
/* Waits for the context's stream; also reports a tensor-core contraction that gave up. */
int champ_synchronize(champ_ctx *ctx);

/* T-moves (tmove.f90:1-192, Casula's size-consistent T-moves; psi_utils_mod.f90:390 do_tmoves) of
   every electron of every walker, in order: the off-diagonal elements of the nonlocal
   pseudopotential to the quadrature points of each centre in range, T(q) = sum over the nonlocal
   channels of w_q (exp(-tau v_l(r)) - 1) P_l(cos theta) psi(x_q)/psi(x), sampled by heat bath
   against weight 1 for staying (positive elements only); variant 1 (casula1) moves the electron
   there, variant 2 (det_balance1, the reference's default) accepts with min(1, forward sum /
   backward sum over the chosen centre's points about the new position).  The points are rotated
   at random per (walker, step, electron).  moved (host [nw] or NULL) receives the accepted
   T-moves per walker.  A DMC run makes them at the start of every step when option "tmoves" is 1
   or 2 (rundmc_mod.f90:137). */
int champ_tmoves(champ_ctx *ctx, uint64_t seed, uint64_t step, double tau, int32_t variant, int32_t *moved);

/* The VMC mover of champ_vmc_sweeps and champ_vmc_run_host (imetro of the reference's control
   menu, control_mod.f90:78-82 and 375-385, default there 6).  imetro 1: Gaussian displacements
   of the step size those calls take (the engine's default).  imetro 6: the accelerated
   Metropolis method of metrop_slat_mov1.f90:82-546 -- each electron moves in spherical
   coordinates about its nearest nucleus, its new radius drawn between r/deltar and r*deltar from a
   Slater-like distribution shaped by the radial drift (and by the nuclear cusp in all-electron
   systems), its polar angle within a cone of 1 - cos(theta) up to deltat + (2 - deltat)/(1 +
   (Z r)^2), its azimuth biased by the tangential drift times fbias, the forward and reverse
   transition probabilities in the acceptance; the step size is then unused.  Out-of-range values
   are corrected as the reference does (deltar < 1 -> 2, deltat outside [0, 2] -> 2, fbias clamped
   to [0, 2]); the reference's defaults are deltar 5, deltat 1, fbias 1.  The random numbers come
   from the same counter-based generator, keyed by (seed, walker, sweep, electron, draw). */
int champ_set_mover(champ_ctx *ctx, int32_t imetro, double deltar, double deltat, double fbias);

/* Engine options (no counterpart in the reference, which has one code path).
   "orbital_tc": 1 computes the orbitals of the full evaluation (value, gradient, Laplacian of
   every electron of every walker) as one tcgen05 tensor-core contraction per spin with a
   3-term TF32 split (about FP32 accuracy), with the basis functions formed in shared memory
   (fused; up to 96 orbitals of a spin, else as 2); 2 the same contraction from basis rows
   written to HBM first; 0 uses the CUDA-core contraction.  Available for
   FP32 precision when the walker state lives in HBM and a spin has >= 16 orbitals, and on by
   default there; CHAMP_EINVAL otherwise.  The calls that run it (champ_set_walkers,
   champ_eval_full, champ_vmc_sweeps, champ_vmc_run_host) synchronise and return CHAMP_ECUDA if
   a contraction gave up waiting for its MMA groups (bounded waits), then clear that flag.
   "orbital_tc_chunk": K-blocks of 16 basis functions that the fused contraction sums into one
   TMEM accumulator before adding it to the orbital rows in FP32 (default 4; 0 = all of K).  The
   tensor core truncates while it accumulates, so shorter chunks shrink the resulting bias
   towards zero of the orbitals (and with it of ln|D| and E_L) at the cost of a read-modify-write
   of the rows per chunk.
   "reinvert_every": the full evaluation after a VMC sweep re-inverts the Slater matrices in
   FP64 every this many sweeps (sweep index divisible by it) and otherwise uses the inverses
   kept current by the Sherman-Morrison updates of the accepted moves; default
   ceil(100 / nelec), i.e. a re-inversion about every 100 single-electron moves.
   "dmc_graph": 1 (default) replays pairs of DMC steps as a captured CUDA graph, 0 launches the
   kernels of every step from the host.
   "phase_timing": 1 records CUDA events around the VMC sweep kernels (champ_phase_times).
   "staged_eval": 1 (default when the walker state of an FP64 or mixed context lives in HBM)
   runs the FP64 full evaluation as four kernels sized for their own parts (Jastrow and
   distances; basis and orbitals per electron; Slater-matrix inversion in shared memory;
   velocities, pseudopotential and E_L), and a VMC sweep of an FP64 context as its moves followed
   by that evaluation; 0 runs the single-kernel evaluation (and the fused FP64 sweep kernel).
   "tmoves": 0 (default), 1 or 2 -- T-moves of the variant of champ_tmoves at the start of every
   DMC step (champ_dmc_steps).
   "dmc_ene_int": 1 (default) ene_int_v9 energy integration in the DMC reweighting, 0 none.
   "move_coop": 1 (default where available: FP32 or mixed single-determinant contexts whose walker
   state lives in HBM, 17 to 128 orbitals per spin) runs the FP32 Gaussian moves with the warps of
   a block sharing the proposals' orbital-coefficient stream through shared memory (cp.async), in
   step electron by electron; 0 lets every warp stream the coefficients itself.  The walks are the
   same.
   "orb_coop": 1 (default where available: the staged evaluation with electrons and up electrons in
   multiples of 4 and more than 16 orbitals per spin) lets the warps of a block of its orbital part
   share the coefficient stream through shared memory; 0 lets every warp stream it.  Same results.
   "mover_cache": 1 (default) lets the accelerated mover of a mixed single-determinant context
   whose walker state lives in HBM take the drift at an electron's current position from the
   orbital rows of the last FP64 evaluation (updated by its accepted moves) instead of evaluating
   the basis functions and orbitals there again; 0 evaluates them.  The two differ at FP32 rounding.
   "dmc_persistent": 1 runs the DMC step kernel persistent (resident blocks taking walkers from a
   work counter), 0 (default) a warp per walker; the results are the same.
   "delay_rank": K >= 2 (default 4 when the walker state of a single-determinant FP64 or mixed
   context lives in HBM) keeps the accepted moves' Sherman-Morrison terms of a spin aside and
   folds K of them at a time into the inverse as one FP64 tensor-core product (proposals use the
   inverse with the pending terms; all are folded in at the end of a sweep's moves); 0 or 1
   applies each update at once. */
int champ_set_option(champ_ctx *ctx, const char *name, int64_t value);
/* Device time of the VMC sweep kernels launched since option "phase_timing" was set to 1 or
   since the previous call (no counterpart in the reference: instrumentation for benchmarks),
   from CUDA events on the context's stream: ms[0] the fused sweep kernel (moves and E_L in one
   launch: FP64 with "staged_eval" 0, and FP32 without the tensor-core orbitals), ms[1] the move
   kernel and ms[2] the FP64 full evaluation of a sweep made of the two (mixed precision, and FP64
   with "staged_eval" 1), ms[3] unused; launches[] (may be NULL) the counts of timed sections.
   Synchronises the stream and resets the sums. */
int champ_phase_times(champ_ctx *ctx, double *ms /* [4] */, int32_t *launches /* [4] or NULL */);
/* Autotuning of the launch shapes (no counterpart in the reference): for the options that change
   only the speed of a VMC sweep -- "delay_rank" (0, 4, 8, 16), "staged_eval" (1, 0), "move_coop"
   (1, 0), "orb_coop" (1, 0), and with the
   tensor-core orbitals of an FP32 context "orbital_tc" (1, 2) and "orbital_tc_chunk" (2, 4, 8) --
   one option at a time, in that order, times nsweep sweeps of the context's walkers (step size
   step, after one untimed sweep; device time from CUDA events) for each value it accepts, and
   keeps the fastest.  The probe sweeps move the walkers as equilibration sweeps would.  With
   cache_path (may be NULL) the choice is appended to that text file under a key of the system's
   shape (electrons, centres, basis functions, orbitals, determinants, e-e-n order, pseudopotential,
   precision, walkers), and a later call with the same key applies it without timing.  report
   (may be NULL) receives a one-line summary: the chosen values and the ms per sweep of each
   candidate. */
int champ_autotune(champ_ctx *ctx, int32_t nsweep, uint64_t seed, double step, const char *cache_path, char *report,
                   int32_t report_len);
/* Current value of an option ("orbital_tc", "orbital_tc_chunk", "reinvert_every", "dmc_graph",
   "phase_timing", "param_grad_mode", "staged_eval", "delay_rank", "tmoves", "dmc_ene_int",
   "dmc_persistent", "move_coop", "orb_coop", "mover_cache"); kernel launches per
   champ_vmc_sweeps sweep
   ("launches_per_sweep": 1 for the fused sweep kernel, 2 for moves + single-kernel evaluation,
   5 for moves + staged evaluation or with the tensor-core orbitals). */
int champ_get_option(const champ_ctx *ctx, const char *name, int64_t *value);

#ifdef __cplusplus
}
#endif

#endif /* CHAMP_B200_H */
