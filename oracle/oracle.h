/*
 * oracle.h -- FP64 CPU restatement of CHAMP's Slater-Jastrow hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it).
 * The engine never links, loads or calls it.
 *
 * Parity status: the reference (Fortran) cannot be compiled in this environment,
 * so this restatement is pinned by the reference's own numerical cross-checks
 * (finite-difference gradients/Laplacians as in qmc/vmc/jastrow_num.f90 and
 * qmc/psi_utils_mod.f90:439,508, tools/test_basis_fns) and by the statistical VMC
 * energies in the reference's example transcripts, not by per-configuration golden
 * vectors (the reference ships none).
 */
#ifndef CHAMP_ORACLE_H
#define CHAMP_ORACLE_H

#include <stdint.h>
#include "../include/champ_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* Results of one full evaluation (hpsi) of one walker. */
typedef struct orc_eval {
  double lnpsi, sign, psij, lnd;
  double d2lnpsi, d2j, d2lnd;
  double pe, pe_ee, pe_local, pe_nonloc, pecent, energy;
  double *vel;    /* [N][3] grad ln psi */
  double *vj;     /* [N][3] grad J */
  double *vd;     /* [N][3] grad ln D */
  double *div_v;  /* [N] */
} orc_eval;

orc_sys *orc_create(const champ_system *sys);
void orc_destroy(orc_sys *s);
int orc_nterms4(int nord);
/* Jastrow e-e-n coefficients after the cusp conditions were applied (nctype x nterms). */
void orc_get_c(const orc_sys *s, double *c);
/* Rotation of the quadrature grid (row-major 3x3, q = R q0); NULL = identity. */
void orc_set_rotation(orc_sys *s, const double *rot);
void orc_quadrature(const orc_sys *s, double *xyzw /* [nquad][4] rotated points + weight */);

/* hpsi for one walker; vel/vj/vd/div_v may be NULL. Returns 0, or 1 if singular. */
int orc_eval_full(const orc_sys *s, const double *x /* [N][3] */, orc_eval *out);

/* Individual pieces, exported for unit tests. */
void orc_basis(const orc_sys *s, const double *r /* point [3] */,
               double *phi /* [nbasis][5]: value, d/dx, d/dy, d/dz, laplacian */);
void orc_orbitals(const orc_sys *s, const double *r, double *orb /* [norb][5] */);
/* jastrow4: value, v[N][3], d2 (sum of laplacians). */
double orc_jastrow(const orc_sys *s, const double *x, double *v, double *d2);
/* Local pseudopotential channel sum and nonlocal-channel values for electron-centre distance r. */
void orc_vps(const orc_sys *s, int ict, double r, double *vps /* [npotd] */);

/* hpsie for one walker: psi(new)/psi(old) with electron iel at xnew, and grad ln psi
   of electron iel at xnew (grad may be NULL). */
double orc_ratio_1e(const orc_sys *s, const double *x, int iel, const double *xnew, double *grad);
/* Free Jastrow parameters (engine order): dJ/dp, d grad J/dp [np][N][3], d sum lap J/dp at x
   (gvel, d2 may be NULL); returns np. */
int orc_jastrow_pderiv(const orc_sys *s, const double *x, double *gval, double *gvel, double *d2);
/* d ln psi/dp and d E_L/dp of the free Jastrow parameters at x; np, or -1 when singular. */
int orc_jastrow_param_grad(const orc_sys *s, const double *x, double *dlnpsi, double *deloc);

/* Counter-based random numbers shared in definition with the engine (Philox4x32-10). */
void orc_philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t *out4);
/* Uniform random rotation for (seed, walker, sweep) (Shoemake quaternion method). */
void orc_random_rotation(uint64_t seed, uint32_t walker, uint64_t sweep, double *rot);

/* VMC on nw walkers with the engine's move sequence: Gaussian proposals of width step,
   Metropolis accept on |psi ratio|^2, full E_L after each sweep with the quadrature
   rotated per (walker, sweep).  Incremental single-electron updates as in
   metrop_mov1/hpsie/jassav/detsav.  x is updated in place.  nthreads <= 0: all cores. */
/* T-moves of every electron of one walker (in place); returns the accepted moves. */
int orc_tmoves(const orc_sys *s, double *x, uint64_t seed, uint32_t iw, uint64_t step, double tau, int variant);
/* VMC with the accelerated Metropolis mover (imetro = 6). */
int orc_vmc_accel(const orc_sys *s, int nw, double *x, int nsweep, uint64_t seed, uint64_t sweep0, double deltar,
                  double deltat, double fbias, double *esum, double *e2sum, double *accept, double *elast,
                  int nthreads);
int orc_vmc(const orc_sys *s, int nw, double *x, int nsweep, uint64_t seed, uint64_t sweep0,
            double step, double *esum, double *e2sum, double *accept, double *elast,
            int nthreads);

#ifdef __cplusplus
}
#endif
#endif
