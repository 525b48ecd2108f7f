// dmc.cuh -- diffusion Monte Carlo step for a varying walker population.
//
// One step (rundmc_mod.f90:123-365): for every walker, every electron makes a drift-diffusion
// proposal x' = x + tau vbar(x) + sqrt(tau) chi with the averaged drift of
// averaged_1e_velocity (green_functions_mod.f90:598-633, n_drift_param = 2), accepted with
// min(1, |psi'/psi|^2 G(x<-x')/G(x'<-x)) (sample_1e_prob), node crossings rejected; then the
// full E_L, and the weight is multiplied by exp(-tau ((E_L,old + E_L,new)/2 - E_T)).
// Branching (split_join, dmc/dmc_elec/split_join_mod.f90): each walker is copied
// floor(w + u) times with weight 1 into a second state buffer (exclusive scan for the
// destinations); the trial energy follows the population: E_T = E_est - ln(W/W_target)/(g tau).
// The walker count lives on the device, so steps need no host synchronisation.
#pragma once

struct DmcPar {
  double tau, adrift, gpop, ecut;
  int wtarget, wmax;
  uint64_t seed;
};

// per-walker DMC data (weights, E_L at the last step) and device scalars
struct DmcData {
  double *wt, *el;        // [wmax]
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

// phase 0: moves, E_L and reweighting in one pass; 1: the moves only; 2: E_L (from the positions,
// re-inverting, refreshing the FP32 move tables when the state has them) and reweighting only --
// the FP32 and FP64 halves of a mixed-precision step.
template <class T, int NORD, bool MD>
__global__ void __launch_bounds__(128, 4) k_dmc_move(Sys<T> s, State<T> st, Layout L, DmcPar P, DmcData D, int phase) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N, W = *D.nw;
  const double et = *D.et, sqt = sqrt(P.tau);
  const uint64_t step = (uint64_t)D.ctr[0];
  for (int w = blockIdx.x * wpb + wib; w < W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, L.resident != 0);
    if (L.resident && phase != 2) {
      view_load(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
    }
    int acc = 0;
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
      if (ua < p) {
        accept_move<T, MD>(s, st, w, v, e, xn, dj, rho, lane);
        acc++;
      }
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
      double eo = D.el[w], en = res.eloc;
      double de = 0.5 * (eo + en) - et;
      de = de > P.ecut ? P.ecut : (de < -P.ecut ? -P.ecut : de);  // reweighting cut-off
      double wn = D.wt[w] * exp(-P.tau * de);
      if (!isfinite(wn) || !isfinite(en)) wn = 0.0;  // a walker with a non-finite energy dies
      D.wt[w] = wn;
      D.el[w] = en;
    }
    __syncwarp();
  }
}

// weights -> copy counts (stochastic rounding); zero beyond the population
static __global__ void k_dmc_count(DmcData D, DmcPar P) {
  const int W = *D.nw;
  const uint64_t step = (uint64_t)D.ctr[0];
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < P.wmax; w += gridDim.x * blockDim.x) {
    int nc = 0;
    if (w < W) {
      uint32_t o[4];
      philox(P.seed, (uint32_t)w, (uint32_t)step, (uint32_t)(step >> 32), 0xFFFFFFFEu, o);
      double u = u53(o[0], o[1]);
      double c = floor(D.wt[w] + u);
      nc = c > 8 ? 8 : (int)c;
    }
    D.ncopy[w] = nc;
  }
}

// sums for the mixed estimator: red[0] = sum w, red[1] = sum w E_L (warp shuffles + atomics)
static __global__ void k_dmc_sums(DmcData D, int wmax) {
  const int W = *D.nw;
  double a = 0, b = 0;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W && w < wmax; w += gridDim.x * blockDim.x) {
    a += D.wt[w];
    b += D.wt[w] * D.el[w];
  }
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&D.red[0], a);
    atomicAdd(&D.red[1], b);
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
  double et = eest - log((tot > 0 ? (double)tot : 1.0) / (double)P.wtarget) / (P.gpop * P.tau);
  *Db.nw = tot;
  *Db.eest = eest;
  *Db.et = et;
  *Da.eest = eest;
  *Da.et = et;
  double *st = Da.stat + 4 * (size_t)istat;
  st[0] = (double)W;
  st[1] = sw;
  st[2] = swe;
  st[3] = et;
  Da.red[0] = 0;
  Da.red[1] = 0;
  Db.red[0] = 0;
  Db.red[1] = 0;
  Da.ctr[0] += 1;
  Da.ctr[1] += 1;
}
