// dmc.cuh -- diffusion Monte Carlo step for a varying walker population.
//
// One step (rundmc_mod.f90:123-365): for every walker, every electron makes a drift-diffusion
// proposal x' = x + tau vbar(x) + sqrt(tau) chi with the averaged drift of
// averaged_1e_velocity (green_functions_mod.f90:598-633, n_drift_param = 2), accepted with
// min(1, |psi'/psi|^2 G(x<-x')/G(x'<-x)) (sample_1e_prob), node crossings rejected; then the
// full E_L, and the weight is multiplied by exp(-tau_eff (E_int - E_T)), with the energy integrated
// over the step as ene_int_rewt does for the default ene_int_v9 (green_functions_mod.f90:382-472):
// each end's E_L - E_est is damped by (sqrt(pi)/2) erf(f)/f, f = |grad ln psi| / sqrt(N) tau_eff c_rewt,
// which removes the locality approximation's negative spikes near the nodes; E_int is floored at
// E_est - limit_rewt_dmc sigma_E / tau^(1/4); tau_eff = tau sum_i p_i chi_i^2 / sum_i chi_i^2 over
// the electrons' acceptance probabilities and diffusion steps (itau_eff = 1, rundmc_mod.f90:203-210).
// Branching (split_join, dmc/dmc_elec/split_join_mod.f90): each walker is copied
// floor(w + u) times with weight 1 into a second state buffer (exclusive scan for the
// destinations); the trial energy follows the population: E_T = E_g - ln(W/W_target)/(g tau),
// E_g a running average of the growth energy.
// The walker count lives on the device, so steps need no host synchronisation.
#pragma once

struct DmcPar {
  double tau, adrift, gpop;
  double rewt_limit, c_rewt;  // limit_rewt_dmc, c_rewt (control_mod.f90:16)
  int ene_int;                // 1: ene_int_v9 (the reference's default), 0: no_ene_int
  int wtarget, wmax;
  uint64_t seed;
  int tmove;  // T-moves before each step's drift-diffusion moves: 0 off, 1 casula1, 2 det_balance1
  int persist;  // step kernel: 1 persistent (work counter), 0 one walker per warp
};

// per-walker DMC data (weights, E_L at the last step) and device scalars
struct DmcData {
  double *wt, *el;        // [wmax]
  double *v2;             // [wmax] |grad ln psi|^2 at the last step
  double *teff;           // [wmax] the step's effective time step (written by the moves)
  double *esg;            // [4] (device) generations, sum sw, sum sw E, sum sw E^2 since the start
  double *egr;            // (device) running growth energy, the reference of the trial energy
  int *next;              // [2] (device) work counters of the persistent step kernel (moves, E_L)
  int *nw;                // current population (device)
  double *et;             // trial energy (device)
  double *eest;           // running estimate of the energy (device)
  int *ncopy, *off;       // [wmax]
  double *stat;           // [nstep][4]: population, sum w, sum w E_L, E_T
  double *red;            // [2] sum w, sum w E_L of the step
  long long *ctr;         // [2] (device) step counter (random-number key), statistics record index
};

// averaged drift (averaged_1e_velocity with n_drift_param = 2)
__device__ __forceinline__ void avg_drift(const double *g, double tau, double a, double *vb) {
  double v2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  double f = 1.0;
  if (a * v2 * tau > 0) f = (-1.0 + sqrt(1.0 + 2.0 * a * v2 * tau)) / (a * v2 * tau);
  vb[0] = f * g[0]; vb[1] = f * g[1]; vb[2] = f * g[2];
}

// sigma of E_L for the reweighting floor (rundmc_mod.f90:238-244): 0.2 sqrt(N) for the first
// max(10, 10/tau) generations, then sqrt(W_target) times the weighted standard deviation of the
// generations' mixed estimators (stats_sigma, stats_type_mod.f90:270-280)
__device__ inline double energy_sigma(const DmcPar &P, const double *esg, int N) {
  const double ngen = esg[0], nmin = fmax(10.0, rint(10.0 / P.tau));
  if (ngen <= nmin || esg[1] <= 0) return 0.2 * sqrt((double)N);
  const double avg = esg[2] / esg[1], var = esg[3] / esg[1] - avg * avg;
  return sqrt((double)P.wtarget) * sqrt(var > 0 ? var : 0.0);
}

// E_int - E_T of one walker's step (ene_int_rewt, green_functions_mod.f90:382-472): the old and new
// local energies, each damped towards E_est by (sqrt(pi)/2) erf(f)/f with
// f = max(|grad ln psi| / N^pow_rewt tau_int c_rewt, 1e-9), pow_rewt = 1/2, tau_int = tau_eff
// (itau_integ = 1); their mean minus E_T, floored at E_est - E_T - limit_rewt_dmc sigma / tau^(1/4).
__device__ inline double integrated_energy(const DmcPar &P, double eo, double v2o, double en, double v2n, int N,
                                           double eest, double et, double esigma, double tauint) {
  double ewo = eo, ewn = en;
  if (P.ene_int == 1) {
    const double spi = 0.886226925452758;  // sqrt(pi) / 2
    const double rn = 1.0 / sqrt((double)N);
    const double fo = fmax(sqrt(v2o) * rn * tauint * P.c_rewt, 1e-9);
    const double fn = fmax(sqrt(v2n) * rn * tauint * P.c_rewt, 1e-9);
    ewo = eest + (eo - eest) * spi * erf(fo) / fo;
    ewn = eest + (en - eest) * spi * erf(fn) / fn;
  }
  const double eint = 0.5 * (ewo + ewn) - et;
  const double emin = eest - et - P.rewt_limit * esigma / sqrt(sqrt(P.tau));
  return eint < emin ? emin : eint;
}

// copies of walker w at branching (split_join): floor(w + u) with u from the walker's stream of
// the step, at most 8
__device__ inline int copy_count(const DmcPar &P, double wt, int w, uint64_t step) {
  uint32_t o[4];
  philox(P.seed, (uint32_t)w, (uint32_t)step, (uint32_t)(step >> 32), 0xFFFFFFFEu, o);
  const double c = floor(wt + u53(o[0], o[1]));
  return c > 8 ? 8 : (int)c;
}

// The DMC step kernel: a warp per walker, or (P.persist) persistent -- resident blocks whose warps
// take walkers from a work counter (D.next) until the population is done.  The persistent form
// measured 1.8x slower on the 8-electron dimer at 35k walkers (adjacent branched copies no longer
// run side by side on one SM), so a warp per walker is the default.  With the reweighting it also
// forms the branching copy counts and the weight sums of the step.
// phase 0: moves, E_L and reweighting in one pass; 1: the moves only; 2: E_L (from the positions,
// re-inverting, refreshing the FP32 move tables when the state has them) and reweighting only --
// the FP32 and FP64 halves of a mixed-precision step.
template <class T, int NORD, bool MD>
__global__ void __launch_bounds__(128, 4) k_dmc_move(Sys<T> s, State<T> st, Layout L, DmcPar P, DmcData D, int phase) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int N = s.N, W = *D.nw;
  const double et = *D.et, eest = *D.eest, sqt = sqrt(P.tau);
  const double esigma = energy_sigma(P, D.esg, N);
  const uint64_t step = (uint64_t)D.ctr[0];
  int *next = D.next + (phase == 2 ? 1 : 0);
  double sw = 0, swe = 0;  // this warp's sums of w and w E_L (lane 0)
  for (int pass = 0;; pass++) {
    int w = 0;
    if (P.persist) {
      if (lane == 0) w = atomicAdd(next, 1);
      w = __shfl_sync(0xffffffffu, w, 0);
    } else {
      w = pass == 0 ? blockIdx.x * (blockDim.x >> 5) + wib : W;
    }
    if (w >= W) break;
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, L.resident != 0);
    if (L.resident && phase != 2) {
      view_load(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
    }
    int acc = 0;
    double sdd = 0, spd = 0;  // sum_i chi_i^2 tau and sum_i p_i chi_i^2 tau over the electrons
    for (int e = 0; e < N && phase != 2; e++) {
      double xo[3] = {v.xs[3 * e], v.xs[3 * e + 1], v.xs[3 * e + 2]};
      double r0, d0, go[3], gn[3], vo[3], vn[3];
      propose<T, NORD, MD, true>(s, J, st, w, v, e, xo, lane, r0, d0, go);  // grad at the current position
      avg_drift(go, P.tau, P.adrift, vo);
      double g[3], ua;
      move_randoms(P.seed, (uint32_t)w, step, (uint32_t)e, g, &ua);
      double xn[3];
      for (int k = 0; k < 3; k++) xn[k] = xo[k] + P.tau * vo[k] + sqt * g[k];
      double rho, dj;
      propose<T, NORD, MD, true>(s, J, st, w, v, e, xn, lane, rho, dj, gn);
      avg_drift(gn, P.tau, P.adrift, vn);
      double lgf = -0.5 * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
      double db[3] = {xo[0] - xn[0] - P.tau * vn[0], xo[1] - xn[1] - P.tau * vn[1], xo[2] - xn[2] - P.tau * vn[2]};
      double lgb = -(db[0] * db[0] + db[1] * db[1] + db[2] * db[2]) / (2 * P.tau);
      double p = (rho > 0) ? rho * rho * exp(2.0 * dj + lgb - lgf) : 0.0;  // fixed node
      const double dd = P.tau * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
      sdd += dd;
      spd += (p < 1.0 ? p : 1.0) * dd;
      if (ua < p) {
        accept_move<T, MD>(s, st, w, v, e, xn, dj, rho, lane);
        acc++;
      }
    }
    double teff = P.tau;
    if (phase != 2) {
      teff = sdd > 0 ? P.tau * spd / sdd : P.tau;
      if (phase == 1 && lane == 0) D.teff[w] = teff;
    } else {
      teff = D.teff[w];
    }
    if (phase == 1) {
      if (L.resident) view_store(v, st, w, N, s.C, lane);
      else {
        for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
        __syncwarp();
      }
      continue;
    }
    double R[9];
    random_rotation(P.seed, (uint32_t)w, step, R);
    EvalRes res;
    full_eval<T, NORD, MD>(s, J, E, st, w, v, R, lane, false, res);
    if (phase == 2) {
      if (L.resident) eval_store(v, st, w, N, s.C, lane);
      else mirror_store(v, st, w, N, s.C, lane);
    } else if (L.resident) view_store(v, st, w, N, s.C, lane);
    else {
      for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
      __syncwarp();
    }
    if (lane == 0) {
      const double eo = D.el[w], en = res.eloc;
      const double eint = integrated_energy(P, eo, D.v2[w], en, res.v2, N, eest, et, esigma, teff);
      double wn = D.wt[w] * exp(-eint * teff);
      if (!isfinite(wn) || !isfinite(en)) wn = 0.0;  // a walker with a non-finite energy dies
      D.wt[w] = wn;
      D.el[w] = en;
      D.v2[w] = res.v2;
      D.ncopy[w] = copy_count(P, wn, w, step);
      sw += wn;
      if (wn > 0) swe += wn * en;
    }
    __syncwarp();
  }
  if (phase == 1) return;
  // the step's sums for the mixed estimator (red[0] = sum w, red[1] = sum w E_L), and no copies
  // beyond the population
  if (lane == 0 && sw != 0) {
    atomicAdd(&D.red[0], sw);
    atomicAdd(&D.red[1], swe);
  }
  const int gw = blockIdx.x * (blockDim.x >> 5) + wib, nwarp = gridDim.x * (blockDim.x >> 5);
  for (int i = W + gw * 32 + lane; i < P.wmax; i += nwarp * 32) D.ncopy[i] = 0;
}

// Uniform random rotation (Shoemake's quaternion method) from three draws of a move's stream.
__device__ inline void rotation_from(MoveRng &rng, double *R) {
  const double u1 = rng.next(), u2 = rng.next(), u3 = rng.next();
  const double tp = 6.283185307179586, s1 = sqrt(1.0 - u1), s2 = sqrt(u1);
  double sa, ca, sb, cb;
  sincos(tp * u2, &sa, &ca);
  sincos(tp * u3, &sb, &cb);
  const double qx = s1 * sa, qy = s1 * ca, qz = s2 * sb, qw = s2 * cb;
  R[0] = 1 - 2 * (qy * qy + qz * qz); R[1] = 2 * (qx * qy - qz * qw); R[2] = 2 * (qx * qz + qy * qw);
  R[3] = 2 * (qx * qy + qz * qw); R[4] = 1 - 2 * (qx * qx + qz * qz); R[5] = 2 * (qy * qz - qx * qw);
  R[6] = 2 * (qx * qz - qy * qw); R[7] = 2 * (qy * qz + qx * qw); R[8] = 1 - 2 * (qx * qx + qy * qy);
}

// T-move of electron e (tmove.f90:1-192, Casula's size-consistent T-moves): the nonlocal
// pseudopotential's off-diagonal elements to the quadrature points of every centre in range,
// T(q) = sum_{l nonlocal} w_q (exp(-tau v_l(r)) - 1) P_l(cos theta) psi(x_q)/psi(x), sampled by heat
// bath against weight 1 for staying (positive T only); with det_balance1 (variant 2) the move is
// then accepted with min(1, sum_forward / sum_backward), the backward sum over the chosen centre's
// points about the new position (fresh rotation).  The point grid is rotated at random per
// (walker, step, electron); the draws come from that move's own stream.  Returns whether the
// electron moved (its state updated as by an accepted single-electron move).
template <class T, int NORD, bool MD>
__device__ bool tmove_electron(const Sys<T> &s, const JasPar<T> &J, const EcpPar &E, const State<T> &st, int w,
                               const View<T> &v, int e, double tau, int variant, uint64_t seed, uint64_t step,
                               int lane) {
  MoveRng rng{seed, (uint32_t)w, (uint32_t)step, (uint32_t)(step >> 32), 256u + (uint32_t)e, 0u, {0.0, 0.0}, 0};
  double R[9];
  rotation_from(rng, R);
  const double xo[3] = {v.xs[3 * e], v.xs[3 * e + 1], v.xs[3 * e + 2]};
  double S = 1.0, pratio = 0.0;
  int pc = -1, pq = -1;
  for (int c = 0; c < s.C; c++) {
    const double *cc = s.cent + 3 * c;
    const double rv[3] = {xo[0] - cc[0], xo[1] - cc[1], xo[2] - cc[2]};
    const double r = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
    const int it = s.ctype[c];
    double vps[MAXLCH];
    ecp_vps(E, it, r, vps);
    bool skip = true;
    for (int l = 0; l < E.npotd[it]; l++)
      if (l + 1 != E.lpotp1[it] && fabs(vps[l]) > 1e-4) skip = false;
    if (skip) continue;
    for (int q = 0; q < E.nquad; q++) {
      double qv[3];
      for (int k = 0; k < 3; k++)
        qv[k] = R[3 * k] * s.quad->q0[q][0] + R[3 * k + 1] * s.quad->q0[q][1] + R[3 * k + 2] * s.quad->q0[q][2];
      const double costh = (rv[0] * qv[0] + rv[1] * qv[1] + rv[2] * qv[2]) / r;
      const double xq[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
      double rho, dj, g[3];
      propose<T, NORD, MD, false>(s, J, st, w, v, e, xq, lane, rho, dj, g);
      const double ratio = rho * exp(dj);
      double gp = 0;
      for (int l = 0; l < E.npotd[it]; l++)
        if (l + 1 != E.lpotp1[it]) gp += s.quad->wq[q] * (exp(-tau * vps[l]) - 1) * yl0(l, costh) * ratio;
      if (gp > 0) {
        S += gp;
        if (rng.next() < gp / S) { pc = c; pq = q; pratio = ratio; }
      }
    }
  }
  if (pc < 0) return false;
  const double *cc = s.cent + 3 * pc;
  const double r = sqrt((xo[0] - cc[0]) * (xo[0] - cc[0]) + (xo[1] - cc[1]) * (xo[1] - cc[1]) +
                        (xo[2] - cc[2]) * (xo[2] - cc[2]));
  double xn[3];
  for (int k = 0; k < 3; k++)
    xn[k] = cc[k] + r * (R[3 * k] * s.quad->q0[pq][0] + R[3 * k + 1] * s.quad->q0[pq][1] +
                         R[3 * k + 2] * s.quad->q0[pq][2]);
  double p = 1.0;
  if (variant == 2) {
    const int it = s.ctype[pc];
    double vps[MAXLCH];
    ecp_vps(E, it, r, vps);
    double R2[9];
    rotation_from(rng, R2);
    const double xe[3] = {xn[0] - cc[0], xn[1] - cc[1], xn[2] - cc[2]};
    double Sb = 1.0;
    for (int q = 0; q < E.nquad; q++) {
      double qv[3];
      for (int k = 0; k < 3; k++)
        qv[k] = R2[3 * k] * s.quad->q0[q][0] + R2[3 * k + 1] * s.quad->q0[q][1] + R2[3 * k + 2] * s.quad->q0[q][2];
      const double costh = (xe[0] * qv[0] + xe[1] * qv[1] + xe[2] * qv[2]) / r;
      const double xq[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
      double rho, dj, g[3];
      propose<T, NORD, MD, false>(s, J, st, w, v, e, xq, lane, rho, dj, g);
      const double ratio = rho * exp(dj) / pratio;
      double gp = 0;
      for (int l = 0; l < E.npotd[it]; l++)
        if (l + 1 != E.lpotp1[it]) gp += s.quad->wq[q] * (exp(-tau * vps[l]) - 1) * yl0(l, costh) * ratio;
      if (gp > 0) Sb += gp;
    }
    p = S / Sb < 1.0 ? S / Sb : 1.0;
  }
  if (rng.next() >= p) return false;
  double rho, dj, g[3];
  propose<T, NORD, MD, false>(s, J, st, w, v, e, xn, lane, rho, dj, g);
  accept_move<T, MD>(s, st, w, v, e, xn, dj, rho, lane);
  return true;
}

// T-moves of every electron of walkers [0, W) (W from *nw when not null): the first part of a DMC
// step with T-moves (rundmc_mod.f90:137, do_tmoves), or on its own (champ_tmoves).  moved (may be
// null) receives the accepted T-moves per walker.
template <class T, int NORD, bool MD>
__global__ void __launch_bounds__(128, 4) k_dmc_tmove(Sys<T> s, State<T> st, Layout L, int W_host, const int *nw,
                                                      double tau, int variant, uint64_t seed, const long long *step_dev,
                                                      uint64_t step_host, int *moved) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N, W = nw ? *nw : W_host;
  const uint64_t step = step_dev ? (uint64_t)step_dev[0] : step_host;
  for (int w = blockIdx.x * wpb + wib; w < W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, L.resident != 0);
    if (L.resident) {
      view_load(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
    }
    int nmv = 0;
    for (int e = 0; e < N; e++) nmv += tmove_electron<T, NORD, MD>(s, J, E, st, w, v, e, tau, variant, seed, step, lane);
    if (L.resident) view_store(v, st, w, N, s.C, lane);
    else {
      for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
      __syncwarp();
    }
    if (moved && lane == 0) moved[w] = nmv;
    __syncwarp();
  }
}

// copy walker w's persistent state (and DMC data) into copies at off[w] ... off[w]+ncopy[w]-1
template <class T>
__global__ void k_dmc_copy(State<T> a, State<T> b, DmcData Da, DmcData Db, int N, int C, int wmax) {
  const int W = *Da.nw;
  const int lane = threadIdx.x & 31, wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
            nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int w = wid; w < W; w += nwarp) {
    int nc = Da.ncopy[w], o0 = Da.off[w];
    for (int c = 0; c < nc; c++) {
      int d = o0 + c;
      if (d >= wmax) break;
      for (int i = lane; i < 3 * N; i += 32) b.x[(size_t)d * 3 * N + i] = a.x[(size_t)w * 3 * N + i];
      for (int i = lane; i < a.astride; i += 32) b.ainv[(size_t)d * a.astride + i] = a.ainv[(size_t)w * a.astride + i];
      for (int i = lane; i < N * N; i += 32) b.fso[(size_t)d * N * N + i] = a.fso[(size_t)w * N * N + i];
      for (int i = lane; i < N * C * 2; i += 32) b.ren[(size_t)d * N * C * 2 + i] = a.ren[(size_t)w * N * C * 2 + i];
      for (int i = lane; i < N * ZQ; i += 32) b.zq[(size_t)d * N * ZQ + i] = a.zq[(size_t)w * N * ZQ + i];
      if (a.rtd)
        for (int i = lane; i < N * C; i += 32) b.rtd[(size_t)d * N * C + i] = a.rtd[(size_t)w * N * C + i];
      for (int i = lane; i < a.tvstride; i += 32) b.tv[(size_t)d * a.tvstride + i] = a.tv[(size_t)w * a.tvstride + i];
      for (int i = lane; i < a.gstride; i += 32) b.gam[(size_t)d * a.gstride + i] = a.gam[(size_t)w * a.gstride + i];
      if (lane == 0) {
        b.fsum[d] = a.fsum[w];
        b.lnd[d] = a.lnd[w];
        b.sgn[d] = a.sgn[w];
        Db.wt[d] = 1.0;
        Db.el[d] = Da.el[w];
        Db.v2[d] = Da.v2[w];
      }
    }
  }
}

// new population, statistics record and trial-energy update (single thread); advances the
// device step counters, so a captured sequence of steps replays with fresh random numbers
static __global__ void k_dmc_finish(DmcData Da, DmcData Db, DmcPar P) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long istat = Da.ctr[1];
  int W = *Da.nw;
  int tot = (W > 0) ? Da.off[P.wmax - 1] + Da.ncopy[P.wmax - 1] : 0;
  if (tot > P.wmax) tot = P.wmax;
  double sw = Da.red[0], swe = Da.red[1];
  double emix = sw > 0 ? swe / sw : *Da.eest;
  // running energy estimate: exponential average of the mixed estimator
  double eest = 0.95 * (*Da.eest) + 0.05 * emix;
  // running growth energy E_T - ln(sum w_new / sum w_old) / tau (every walker enters a step with
  // weight 1, so sum w_old is the population): the trial energy is set from it, so that the
  // population settles at the target even where the integrated energy that drives the weights,
  // damped near the nodes, differs from the mixed estimator of E_L
  if (sw > 0 && W > 0) *Da.egr = 0.95 * (*Da.egr) + 0.05 * (*Da.et - log(sw / (double)W) / P.tau);
  double et = *Da.egr - log((tot > 0 ? (double)tot : 1.0) / (double)P.wtarget) / (P.gpop * P.tau);
  *Db.nw = tot;
  *Db.eest = eest;
  *Db.et = et;
  *Da.eest = eest;
  *Da.et = et;
  if (sw > 0) {  // the generation's mixed estimator, for sigma_E (stats_accuest)
    Da.esg[0] += 1.0;
    Da.esg[1] += sw;
    Da.esg[2] += swe;
    Da.esg[3] += sw * emix * emix;
  }
  double *st = Da.stat + 4 * (size_t)istat;
  st[0] = (double)W;
  st[1] = sw;
  st[2] = swe;
  st[3] = et;
  Da.red[0] = Da.red[1] = 0;
  Db.red[0] = Db.red[1] = 0;
  Da.next[0] = Da.next[1] = 0;
  Da.ctr[0] += 1;
  Da.ctr[1] += 1;
}
