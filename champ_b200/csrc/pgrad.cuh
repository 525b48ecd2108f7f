// pgrad.cuh -- Jastrow parameter derivatives of ln psi and E_L for every walker.
//
// For each Jastrow parameter p the log-derivative g_p = d ln psi / dp is the parameter's
// basis function summed over all e-e, e-n and e-e-n terms (gvalue of
// qmc/vmc/deriv_jastrow4.f90), and
//   dE_L/dp = -1/2 sum_e (lap_e g_p + 2 grad_e ln psi . grad_e g_p) + dV_NL/dp
// (denergy, qmc/vmc/hpsi.f90:357-376), where dV_NL/dp is the nonlocal quadrature weighted
// by the change of g_p when the electron moves to each quadrature point
// (qmc/fit/deriv_nonloc.f90).  The asymptotic constants subtracted from the e-e and e-n
// terms depend on the parameters too, and their derivatives are included.
#pragma once

// basis functions of the e-e parameters b2..b_{nordb+1} for one pair: value t, and with
// DERIV the chain-ruled pieces T1 = t'(r)/r and T2 = t''(r)
template <class T>
__device__ __forceinline__ void ee_param_terms(const JasPar<T> &J, int isb, T ss, T rij, T deni, int k, T &t, T &T1,
                                               T &T2, bool deriv) {
  const T sk = J.scalek, ar = T(1) / sk;
  T u = rij * deni;
  T tu, tuu;
  if (k == 1) {
    T b1 = J.b[isb][0], b2 = J.b[isb][1];
    T bu = T(1) + b2 * u, ba = T(1) + b2 * ar;
    t = -ss * b1 * (u * u / (bu * bu) - ar * ar / (ba * ba));
    tu = -ss * b1 * 2 * u / (bu * bu * bu);
    tuu = -ss * b1 * 2 * (T(1) - 2 * b2 * u) / (bu * bu * bu * bu);
  } else {
    T up = ipow(u, k - 2);
    t = up * u * u - ipow(ar, k);
    tu = T(k) * up * u;
    tuu = T(k * (k - 1)) * up;
  }
  if (deriv) {
    T dd1 = deni * deni, dd2 = -2 * sk * deni * dd1;
    T1 = tu * dd1 / rij;
    T2 = tuu * dd1 * dd1 + tu * dd2;
  }
}

// basis function of the e-n parameter a_{k+1} (k = 2..norda): rr^k - ar^k
template <class T>
__device__ __forceinline__ void en_param_terms(const JasPar<T> &J, T r, T deni, int k, T &t, T &T1, T &T2, bool deriv) {
  const T sk = J.scalek, ar = T(1) / sk;
  T rr = r * deni;
  T p = ipow(rr, k - 2);
  t = p * rr * rr - ipow(ar, k);
  if (deriv) {
    T tr = T(k) * p * rr, trr = T(k * (k - 1)) * p;
    T dd7 = deni * deni, dd9 = -2 * sk * deni * dd7;
    T1 = tr * dd7 / r;
    T2 = trr * dd7 * dd7 + tr * dd9;
  }
}

// Adds one point's contribution to the NLPP parameter sum dvn[idx]: into this lane's slot of
// pg.dvl when the context gave the warp those slots (every lane of the warp adds to the same
// parameters, so atomics serialise 32-fold; the slots are summed into dvn after the quadrature
// loop), else a shared-memory atomic (large FP64 systems, where the slots' shared memory would
// cost more L1 for the kernel's register spills than the atomics cost).
// (The choice is a template parameter, which lets the compiler keep a slot in a register across
// the loop that adds to it.)
template <bool SLOTS>
__device__ __forceinline__ void padd(double *slot, double *dvn, int idx, double v) {
  if (SLOTS) slot[32 * idx] += v;
  else atomicAdd(&dvn[idx], v);
}

// Parameter basis functions with electron e at the quadrature point xn, weighted by coeff
// and added to pg.dvn (through padd).
template <class T, int NORD, bool SLOTS>
__device__ void point_param_values(const Sys<T> &s, const JasPar<T> &J, const View<T> &v, int e, const double *xn,
                                   double coeff, const PGBuf &pg, const T *tsum_pre) {
  const int N = s.N, C = s.C;
  const T sk = J.scalek;
  double *const slot = pg.dvl ? pg.dvl + (threadIdx.x & 31) : nullptr, *const dvn = pg.dvn;
  constexpr Terms tl = make_terms(NORD);
  const bool fast = (NORD > 1) && J.nct == 1 && C <= MAXC_NL;
  const bool xsums = fast && tsum_pre == nullptr;  // e-e-n sums still to form here
  T pr[2 * MAXC_NL], asum[ZQ];
  for (int q = 0; q < ZQ; q++) asum[q] = (q == 0) ? T(C) : T(0);
  for (int c = 0; c < C; c++) {
    T r, d;
    cen_dist(s, sk, xn, c, r, d);
    int it = s.ctype[c];
    for (int k = 2; k <= J.norda; k++) {
      T t, t1, t2;
      en_param_terms(J, r, d, k, t, t1, t2, false);
      padd<SLOTS>(slot, dvn, it * (J.norda - 1) + (k - 2), coeff * (double)t);
    }
    if (xsums) {
      pr[2 * c] = r;
      pr[2 * c + 1] = d;
      T p = d;
      for (int q = 1; q < ZQ; q++) { asum[q] += p; p *= d; }
    }
  }
  T tsum[tl.n > 0 ? tl.n : 1];
#pragma unroll
  for (int ll = 0; ll < tl.n; ll++) tsum[ll] = T(0);
  for (int j = 0; j < N; j++) {
    if (j == e) continue;
    int isb, ipar;
    T ss;
    pair_class(J, s.nup, e, j, isb, ss, ipar);
    const double *xj = v.xs + 3 * j;
    T a0 = T(xn[0] - xj[0]), a1 = T(xn[1] - xj[1]), a2 = T(xn[2] - xj[2]);
    T rij = tsqrt(a0 * a0 + a1 * a1 + a2 * a2);
    T du = T(1) / (T(1) + sk * rij);
    for (int k = 1; k <= J.nordb; k++) {
      T t, t1, t2;
      ee_param_terms(J, isb, ss, rij, du, k, t, t1, t2, false);
      padd<SLOTS>(slot, dvn, pg.na + isb * J.nordb + (k - 1), coeff * (double)t);
    }
    if (xsums) {
      T X[make_mixed(NORD).n > 0 ? make_mixed(NORD).n : 1];
      een_xsums<T, NORD>(C, pr + 1, 2, v.ren + 2 * C * j + 1, 2, X);
      const T *zj = v.zq + ZQ * j;
      constexpr XIdx xi = make_xidx(NORD);
      T uu[NORD + 1];
      uu[0] = T(1);
#pragma unroll
      for (int q = 1; q <= NORD; q++) uu[q] = uu[q - 1] * du;
#pragma unroll
      for (int ll = 0; ll < tl.n; ll++)
        tsum[ll] += uu[tl.k[ll]] * (xsel(xi.a1[ll], asum, zj, X) + xsel(xi.a2[ll], asum, zj, X));
    } else if (!fast && NORD > 1) {
      const T *rj_ = v.ren + 2 * C * j;
      for (int c = 0; c < C; c++) {
        T ri, di;
        cen_dist(s, sk, xn, c, ri, di);
        T rj1 = rj_[2 * c + 1];
        T uu[NORD + 1], pi[NORD + 1], pj[NORD + 1];
        uu[0] = pi[0] = pj[0] = T(1);
#pragma unroll
        for (int q = 1; q <= NORD; q++) { uu[q] = uu[q - 1] * du; pi[q] = pi[q - 1] * di; pj[q] = pj[q - 1] * rj1; }
        const int dst = pg.na + pg.nb + s.ctype[c] * tl.n;
#pragma unroll
        for (int ll = 0; ll < tl.n; ll++) {
          const int k = tl.k[ll], l = tl.l[ll], m = tl.m[ll];
          T sl = (l == 0) ? T(2) : pi[l] + pj[l];
          padd<SLOTS>(slot, dvn, dst + ll, coeff * (double)(uu[k] * sl * pi[m] * pj[m]));
        }
      }
    }
  }
  if (fast) {
#pragma unroll
    for (int ll = 0; ll < tl.n; ll++)
      padd<SLOTS>(slot, dvn, pg.na + pg.nb + ll, coeff * (double)(tsum_pre ? tsum_pre[ll] : tsum[ll]));
  }
}

// g_p, K_p = sum_e (lap_e g_p + 2 v_e . grad_e g_p) and old[e][p] for all Jastrow
// parameters (deriv_jastrow4.f90), warp-cooperative; v = pg.vt.
// Pairs are visited as (i, (i + d) mod N), d = 1..N/2 (at d = N/2 for even N only i < N/2),
// lanes along (d, i) with i fastest: when 32 divides N the lanes of one warp instruction have
// distinct i and distinct j, so the per-electron sums old[i][p], old[j][p] take uncontended
// shared-memory atomics (a few lanes share an electron for small N); the K sums
// accumulate in registers and are reduced over the warp once, and G = (1/2) sum_e old[e][p]
// for pair parameters (sum_e old[e][p] for e-n parameters).  With several centre types the
// e-e-n sums are flushed per centre.
template <class T, int NORD>
__device__ void jastrow_param_pass(const Sys<T> &s, const JasPar<T> &J, const View<T> &v, const PGBuf &pg, int lane) {
  const int N = s.N, C = s.C, P = pg.P, half = N / 2;
  const T sk = J.scalek;
  constexpr Terms tl = make_terms(NORD);
  // e-e parameters b_{k+1}, k = 1..nordb, per b set
  {
    double kb0[MAXORD], kb1[MAXORD];
#pragma unroll
    for (int k = 0; k < MAXORD; k++) kb0[k] = kb1[k] = 0.0;
    for (int t = lane; t < half * N; t += 32) {
        const int d = t / N + 1, i = t - (d - 1) * N;
        if (2 * d == N && i >= half) continue;
        const int j = i + d < N ? i + d : i + d - N;
        const double *xi = v.xs + 3 * i, *xj = v.xs + 3 * j;
        const double *vi = pg.vt + 3 * i, *vj = pg.vt + 3 * j;
        int isb, ipar;
        T ss;
        pair_class(J, s.nup, i, j, isb, ss, ipar);
        double rvd[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
        T rij = tsqrt(T(rvd[0] * rvd[0] + rvd[1] * rvd[1] + rvd[2] * rvd[2]));
        T du = T(1) / (T(1) + sk * rij);
        double dv_rv = (vi[0] - vj[0]) * rvd[0] + (vi[1] - vj[1]) * rvd[1] + (vi[2] - vj[2]) * rvd[2];
#pragma unroll
        for (int k = 1; k < MAXORD; k++) {
          if (k > J.nordb) break;
          T t, t1, t2;
          ee_param_terms(J, isb, ss, rij, du, k, t, t1, t2, true);
          const int ip = pg.na + isb * J.nordb + (k - 1);
          const double kk = 2.0 * ((double)t2 + 2.0 * (double)t1) + 2.0 * (double)t1 * dv_rv;
          if (isb) kb1[k - 1] += kk; else kb0[k - 1] += kk;
          atomicAdd(&pg.old[i * P + ip], (double)t);
          atomicAdd(&pg.old[j * P + ip], (double)t);
        }
      }
#pragma unroll
    for (int k = 1; k < MAXORD; k++) {
      double a0 = warp_sum(kb0[k - 1]), a1 = warp_sum(kb1[k - 1]);
      if (lane == 0 && k <= J.nordb) {
        pg.K[pg.na + (k - 1)] += a0;
        if (J.nspin2b > 1) pg.K[pg.na + J.nordb + (k - 1)] += a1;
      }
    }
  }
  if (NORD > 1) {
    double kc[tl.n > 0 ? tl.n : 1];
#pragma unroll
    for (int ll = 0; ll < tl.n; ll++) kc[ll] = 0.0;
    for (int t = lane; t < half * N; t += 32) {
        const int d = t / N + 1, i = t - (d - 1) * N;
        if (2 * d == N && i >= half) continue;
        const int j = i + d < N ? i + d : i + d - N;
        const double *xi = v.xs + 3 * i, *xj = v.xs + 3 * j;
        const double *vi = pg.vt + 3 * i, *vj = pg.vt + 3 * j;
        double rvd[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
        T rij = tsqrt(T(rvd[0] * rvd[0] + rvd[1] * rvd[1] + rvd[2] * rvd[2]));
        T du = T(1) / (T(1) + sk * rij);
        const T *ri_ = v.ren + 2 * C * i, *rj_ = v.ren + 2 * C * j;
        // the values' sums over the centres in the compute precision, added to the FP64 totals
        // once per pair; the K terms (Laplacian and velocity products, which cancel between
        // centres) are accumulated in FP64 term by term
        constexpr bool PP = false;
        T ocp[tl.n > 0 ? tl.n : 1], kcp[PP && tl.n > 0 ? tl.n : 1];
#pragma unroll
        for (int ll = 0; ll < tl.n; ll++) ocp[ll] = T(0);
        if (PP)
#pragma unroll
          for (int ll = 0; ll < tl.n; ll++) kcp[ll] = T(0);
        const T vi0 = T(vi[0]), vi1 = T(vi[1]), vi2 = T(vi[2]), vj0 = T(vj[0]), vj1 = T(vj[1]), vj2 = T(vj[2]);
        const T vi_rv = vi0 * T(rvd[0]) + vi1 * T(rvd[1]) + vi2 * T(rvd[2]);
        const T vj_rv = vj0 * T(rvd[0]) + vj1 * T(rvd[1]) + vj2 * T(rvd[2]);
        for (int c = 0; c < C; c++) {
          const double *cc = s.cent + 3 * c;
          T ri = ri_[2 * c], di = ri_[2 * c + 1], rj = rj_[2 * c], dj = rj_[2 * c + 1];
          const T vi_ri = vi0 * T(xi[0] - cc[0]) + vi1 * T(xi[1] - cc[1]) + vi2 * T(xi[2] - cc[2]);
          const T vj_rj = vj0 * T(xj[0] - cc[0]) + vj1 * T(xj[1] - cc[1]) + vj2 * T(xj[2] - cc[2]);
          // power tables with two zero entries below 0, as in jas_een
          T uu[NORD + 3], rri[NORD + 3], rrj[NORD + 3];
          uu[0] = uu[1] = rri[0] = rri[1] = rrj[0] = rrj[1] = T(0);
          uu[2] = rri[2] = rrj[2] = T(1);
#pragma unroll
          for (int q = 1; q <= NORD; q++) {
            uu[q + 2] = uu[q + 1] * du;
            rri[q + 2] = rri[q + 1] * di;
            rrj[q + 2] = rrj[q + 1] * dj;
          }
          T dd1 = -sk * du * du, dd7 = -sk * di * di, dd8 = -sk * dj * dj;
          T dd2 = 2 * sk * sk * du * du * du, dd9 = 2 * sk * sk * di * di * di, dd10 = 2 * sk * sk * dj * dj * dj;
          T sp = ri + rj, tm = ri - rj;
          T cpst = (rij * rij + sp * tm) / (ri * rij), cmst = (rij * rij - sp * tm) / (rj * rij);
#pragma unroll
          for (int ll = 0; ll < tl.n; ll++) {
            const int k = tl.k[ll], l = tl.l[ll], m = tl.m[ll];
            T ssl = (l == 0) ? T(2) : rri[l + 2] + rrj[l + 2];
            T st = ssl * rri[m + 2] * rrj[m + 2];
            T pi_ = T(l + m) * rri[l + m + 1] * rrj[m + 2] + T(m) * rri[m + 1] * rrj[l + m + 2];
            T pj_ = T(l + m) * rrj[l + m + 1] * rri[m + 2] + T(m) * rrj[m + 1] * rri[l + m + 2];
            T pii = T((l + m) * (l + m - 1)) * rri[l + m] * rrj[m + 2] + T(m * (m - 1)) * rri[m] * rrj[l + m + 2];
            T pjj = T((l + m) * (l + m - 1)) * rrj[l + m] * rri[m + 2] + T(m * (m - 1)) * rrj[m] * rri[l + m + 2];
            T fc = uu[k + 2] * st;
            T fu = T(k) * uu[k + 1] * st, fuu = T(k * (k - 1)) * uu[k] * st;
            T fi = uu[k + 2] * pi_, fj = uu[k + 2] * pj_, fii = uu[k + 2] * pii, fjj = uu[k + 2] * pjj;
            T fui = T(k) * uu[k + 1] * pi_, fuj = T(k) * uu[k + 1] * pj_;
            fuu = fuu * dd1 * dd1 + fu * dd2;
            fui = fui * dd1 * dd7;
            fuj = fuj * dd1 * dd8;
            fii = fii * dd7 * dd7 + fi * dd9;
            fjj = fjj * dd8 * dd8 + fj * dd10;
            fu = fu * dd1 / rij;
            fi = fi * dd7 / ri;
            fj = fj * dd8 / rj;
            const T kk = 2 * (2 * fu + fi + fj) + 2 * fuu + fii + fjj + fui * cpst + fuj * cmst +
                         2 * (fi * vi_ri + fu * vi_rv + fj * vj_rj - fu * vj_rv);
            if (PP) kcp[ll] += kk;
            else kc[ll] += (double)kk;
            ocp[ll] += fc;
          }
          if (J.nct > 1) {  // each centre type has its own c set
            const int base = pg.na + pg.nb + s.ctype[c] * tl.n;
#pragma unroll
            for (int ll = 0; ll < tl.n; ll++) {
              atomicAdd(&pg.K[base + ll], kc[ll] + (PP ? (double)kcp[ll] : 0.0));
              atomicAdd(&pg.old[i * P + base + ll], (double)ocp[ll]);
              atomicAdd(&pg.old[j * P + base + ll], (double)ocp[ll]);
              kc[ll] = 0.0;
              ocp[ll] = T(0);
              if (PP) kcp[ll] = T(0);
            }
          }
        }
        if (J.nct == 1) {
          const int base = pg.na + pg.nb;
#pragma unroll
          for (int ll = 0; ll < tl.n; ll++) {
            if (PP) kc[ll] += (double)kcp[ll];
            atomicAdd(&pg.old[i * P + base + ll], (double)ocp[ll]);
            atomicAdd(&pg.old[j * P + base + ll], (double)ocp[ll]);
          }
        }
      }
    if (J.nct == 1) {
#pragma unroll
      for (int ll = 0; ll < tl.n; ll++) {
        double a = warp_sum(kc[ll]);
        if (lane == 0) pg.K[pg.na + pg.nb + ll] += a;
      }
    }
  }
  // e-n parameters: lanes along electrons, centres in registers
  {
    double ot[MAXORD], kt[MAXORD];
    for (int i = lane; i < N; i += 32) {
#pragma unroll
      for (int k = 0; k < MAXORD; k++) ot[k] = kt[k] = 0.0;
      const double *xi = v.xs + 3 * i, *vi = pg.vt + 3 * i;
      for (int c = 0; c < C; c++) {
        const double *cc = s.cent + 3 * c;
        T r = v.ren[2 * (i * C + c)], d = v.ren[2 * (i * C + c) + 1];
        double v_r = vi[0] * (xi[0] - cc[0]) + vi[1] * (xi[1] - cc[1]) + vi[2] * (xi[2] - cc[2]);
#pragma unroll
        for (int k = 2; k < MAXORD; k++) {
          if (k > J.norda) break;
          T t, t1, t2;
          en_param_terms(J, r, d, k, t, t1, t2, true);
          ot[k - 2] += (double)t;
          kt[k - 2] += (double)(t2 + 2 * t1) + 2.0 * (double)t1 * v_r;
        }
        if (J.nct > 1 || c == C - 1) {  // flush: per centre with several types, else once
          const int it = s.ctype[c];
#pragma unroll
          for (int k = 2; k < MAXORD; k++) {
            if (k > J.norda) break;
            const int ip = it * (J.norda - 1) + (k - 2);
            pg.old[i * P + ip] += ot[k - 2];
            atomicAdd(&pg.K[ip], kt[k - 2]);
            ot[k - 2] = kt[k - 2] = 0.0;
          }
        }
      }
    }
  }
  __syncwarp();
  // G from the per-electron sums: pair parameters are counted on both electrons of the pair
  for (int p = lane; p < P; p += 32) {
    double g = 0;
    for (int e = 0; e < N; e++) g += pg.old[e * P + p];
    pg.G[p] = p < pg.na ? g : 0.5 * g;
  }
  __syncwarp();
}

// Per-walker derivative output: free Jastrow parameters (a, b, then c with the cusp
// dependences folded in), written as d ln psi / dp and dE_L / dp.
struct PGOut {
  double *dlnpsi;  // [W][nfree]
  double *deloc;   // [W][nfree]
  double *eloc;    // [W]
  int nfree;
  double *scr;     // per-walker scratch of the CSF/orbital part (null when there is none)
  size_t scr_stride;
  int part;        // 1: E_L, Jastrow derivatives, local B; 2: CSF and orbital derivatives;
                   // 3: forward pass (E_L, local B, tape); 4: backward pass (Jastrow derivatives)
  int lanesum;     // per-lane slots for the NLPP parameter sums (see padd)
  // tape of the forward pass: per walker the velocities and per-electron point-coefficient sums
  // ([W][4N]), the number of nonlocal tasks ([W]), the task records ([W][N*C][NLT], the
  // evaluation's own) and each point's coefficient ([W][N*C][nquad])
  double *tape_v;
  int *tape_n;
  const double *tape_nlt;
  double *tape_c;
};

// dE_L/dp from the accumulated sums (K -> -1/2 K + the nonlocal part) and the outputs of the
// free Jastrow parameters: a, b as they are, c through the cusp projection (checkdepend4).
template <class T, int NORD>
__device__ void pg_finish(const Sys<T> &s, const JasPar<T> &J, const PGBuf &pg, const PGOut &out, int w, int lane,
                          bool MDcsf) {
  const int N = s.N, P = pg.P, na = pg.na, nb = pg.nb, nt = make_terms(NORD).n;
  for (int p = lane; p < P; p += 32) {
    double dv = pg.dvn[p];
    for (int e = 0; e < N; e++) dv -= pg.csum[e] * pg.old[e * P + p];
    pg.K[p] = -HB * pg.K[p] + dv;
  }
  __syncwarp();
  // output order: CSF, orbital rotations, Jastrow (as deriv_mod.f90:120-247 concatenates them)
  double *ol = out.dlnpsi + (size_t)w * out.nfree, *oe = out.deloc + (size_t)w * out.nfree;
  const int jo = (MDcsf && s.ncsf > 1 ? s.ncsf - 1 : 0) + s.norbp;
  ol += jo;
  oe += jo;
  for (int f = lane; f < out.nfree - jo; f += 32) {
    double g, d;
    if (f < na + nb) {
      g = pg.G[f];
      d = pg.K[f];
    } else {
      int fc = f - na - nb, it = fc / s.ncfree, jf = fc - it * s.ncfree;
      g = 0;
      d = 0;
      for (int ll = 0; ll < nt; ll++) {
        double pm = s.cproj[ll * s.ncfree + jf];
        g += pm * pg.G[na + nb + it * nt + ll];
        d += pm * pg.K[na + nb + it * nt + ll];
      }
    }
    ol[f] = g;
    oe[f] = d;
  }
  __syncwarp();
}

// CSF and orbital-rotation derivatives from the orbital-resolved local energy
// B[e][m] = -1/2 (lap phi_m + 2 v_J . grad phi_m + ddjas phi_m) + V_loc/N phi_m + V_NL,m
// (elocal_orb_bld, deriv_fast_mod.f90:174-209).  Per spin: T = Ainv Atilde and
// dT = Ainv B - (Ainv B)_ref T over all orbitals (dt_bld, :400), E_ref = tr (Ainv B)_ref.
// CSF: dlnpsi = sum_K c_K D_K/psi_D, dE_L = sum_K c_K (D_K/psi_D)(E_K - E_L) with
// E_K = E_ref + tr(alpha_K^-1 dalpha_K) per spin (alpha_deloc_bld :468, csf_derivs_bld :781).
// Orbital rotation i -> j (single determinant): dlnpsi = sum_spin T[i][j], dE_L = sum_spin dT[i][j]
// (dpsi_orb_bld / deloc_orb_bld, deriv_orb_mod.f90:1486,1557).
// Scratch of the multi-determinant orbital tables after the single-determinant part
// [N*B phis][N*5*M orbitals][N*M B][2*nmax*M T][2*nmax*M dT][nmax^2][ndu delo]: per spin
// G At and G B + dG At over the spin's orbital set (2 x [nomax][M] each), dY, dG (2 x [nomax][nmax]
// each), one [nomax][nmax] work matrix and the local-energy-weighted determinant sums ([ndu]).
template <class T>
__device__ __forceinline__ size_t md_ga_offset(const Sys<T> &s) {
  const size_t N = s.N, B = s.nbasis, M = s.norb, nm = s.nmax;
  return N * B + N * 5 * M + N * M + 4 * nm * M + nm * nm + (size_t)(s.ndu[0] + s.ndu[1]);
}

// dY, dG and the orbital tables of a multi-determinant wave function (dy_bld, dg_bld,
// deriv_fast_mod.f90:648-779).  With c_I = sum over determinants K containing unique
// determinant I of c_K w_K (w = product of the spin determinants' signed alpha determinants) and
// cE_I the same sum weighted by the determinant's local-energy delta (delo_up + delo_dn):
//   dY[p][h] = (1/chi) sum_I (cE_I inv_I - c_I inv_I dalpha_I inv_I)[p][h] - esum Y[p][h],
//   esum = sum_spin sum Y[p][k] dT[k][p],
//   dG = (dY - G B_ref - [ref rows] (T_v dY + dT_v Y)) Ainv.
template <class T>
__device__ void md_orbital_tables(const Sys<T> &s, const View<T> &v, int lane, double *scr, double chi, double eref) {
  const int N = s.N, M = s.norb, nmax = s.nmax, nomax = s.nomax, nd0 = s.ndu[0], nd1 = s.ndu[1];
  const double *orbA = scr + (size_t)N * s.nbasis, *Bm = orbA + (size_t)N * 5 * M;
  const double *dTa = Bm + (size_t)N * M + (size_t)2 * nmax * M;
  const double *delo = dTa + (size_t)2 * nmax * M + (size_t)nmax * nmax;
  double *GA = scr + md_ga_offset(s), *GH = GA + (size_t)2 * nomax * M;
  double *dY = GH + (size_t)2 * nomax * M, *dG = dY + (size_t)2 * nomax * nmax, *aux = dG + (size_t)2 * nomax * nmax;
  double *cE = aux + (size_t)nomax * nmax;
  const double *wd = v.wdet, *wg = v.wdet + nd0 + nd1;
  (void)eref;
  // cE per unique determinant of each spin
  for (int i = lane; i < nd0 + nd1; i += 32) cE[i] = 0.0;
  for (int i = lane; i < 2 * nomax * nmax; i += 32) dY[i] = 0.0;
  __syncwarp();
  for (int K = lane; K < s.ndet; K += 32) {
    int iu = s.ciu[K], id = s.cid[K];
    double t = s.ccoef[K] * wd[iu] * wd[nd0 + id] * (delo[iu] + delo[nd0 + id]);
    atomicAdd(&cE[iu], t);
    atomicAdd(&cE[nd0 + id], t);
  }
  __syncwarp();
  const double ichi = 1.0 / chi;
  double esum = 0;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, nv = s.nvirt[sp];
    const double *Y = v.ymd + (sp ? s.nup * s.nvirt[0] : 0), *dTs = dTa + (size_t)sp * nmax * M;
    for (int i = lane; i < nv * n; i += 32) {
      int p = i / n, k = i - p * n;
      esum += Y[i] * dTs[(size_t)k * M + s.occo[sp][n + p]];
    }
  }
  esum = warp_sum(esum);
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, nv = s.nvirt[sp], no = s.nocc[sp];
    if (n == 0) continue;
    const double *dTs = dTa + (size_t)sp * nmax * M;
    double *dYs = dY + (size_t)sp * nomax * nmax;  // [nv][n] (virtual rows)
    for (int I = lane; I < s.ndu[sp]; I += 32) {
      double a[16], inv[16], da[16], t1[16];
      int k = load_alpha(s, v, sp, I, a);
      if (k == 0) continue;
      small_det_inv(a, k, inv);
      const double cI = wg[(sp ? nd0 : 0) + I], cEI = cE[(sp ? nd0 : 0) + I];
      for (int ia = 0; ia < k; ia++)
        for (int ib = 0; ib < k; ib++) da[ia * k + ib] = dTs[(size_t)s.dh[sp][4 * I + ia] * M + s.occo[sp][n + s.dpart[sp][4 * I + ib]]];
      // t1 = inv da inv (inv rows: particles, columns: holes; da rows: holes, columns: particles)
      for (int ib = 0; ib < k; ib++)
        for (int ia = 0; ia < k; ia++) {
          double acc = 0;
          for (int x = 0; x < k; x++)
            for (int y = 0; y < k; y++) acc += inv[ib * k + x] * da[x * k + y] * inv[y * k + ia];
          t1[ib * k + ia] = acc;
        }
      for (int ib = 0; ib < k; ib++)
        for (int ia = 0; ia < k; ia++)
          atomicAdd(&dYs[s.dpart[sp][4 * I + ib] * n + s.dh[sp][4 * I + ia]],
                    (cEI * inv[ib * k + ia] - cI * t1[ib * k + ia]) * ichi);
    }
    __syncwarp();
    const double *Y = v.ymd + (sp ? s.nup * s.nvirt[0] : 0);
    for (int i = lane; i < nv * n; i += 32) dYs[i] -= esum * Y[i];
    __syncwarp();
    // aux = dY - G B_ref - [ref rows] (T_v dY + dT_v Y), then dG = aux Ainv
    const double *G = v.gam + (sp ? s.nocc[0] * s.nup : 0), *A = v.ainv + (sp ? s.nup * s.nup : 0);
    const double *Tv = v.tv + (sp ? s.nup * s.nvirt[0] : 0);
    const int e0 = sp ? s.nup : 0;
    double *dGs = dG + (size_t)sp * nomax * nmax;
    for (int i = lane; i < no * n; i += 32) {
      int o = i / n, kk = i - o * n;
      double acc = o >= n ? dYs[(o - n) * n + kk] : 0.0;
      const int rk = s.occo[sp][kk];
      for (int e = 0; e < n; e++) acc -= G[o * n + e] * Bm[(size_t)(e0 + e) * M + rk];
      if (o < n) {
        for (int p = 0; p < nv; p++)
          acc -= Tv[o * nv + p] * dYs[p * n + kk] + dTs[(size_t)o * M + s.occo[sp][n + p]] * Y[p * n + kk];
      }
      aux[i] = acc;
    }
    __syncwarp();
    for (int i = lane; i < no * n; i += 32) {
      int o = i / n, e = i - o * n;
      double acc = 0;
      for (int kk = 0; kk < n; kk++) acc += aux[o * n + kk] * A[kk * n + e];
      dGs[i] = acc;
    }
    __syncwarp();
    double *GAs = GA + (size_t)sp * nomax * M, *GHs = GH + (size_t)sp * nomax * M;
    for (int i = lane; i < no * M; i += 32) {
      int o = i / M, m = i - o * M;
      double ga = 0, gh = 0;
      for (int e = 0; e < n; e++) {
        double at = orbA[(size_t)(e0 + e) * 5 * M + m];
        ga += G[o * n + e] * at;
        gh += G[o * n + e] * Bm[(size_t)(e0 + e) * M + m] + dGs[o * n + e] * at;
      }
      GAs[i] = ga;
      GHs[i] = gh;
    }
    __syncwarp();
  }
}

// Orbital-resolved local energy (elocal_orb_bld, deriv_fast_mod.f90:174-210), local part:
// orbitals of all M orbitals with gradient and Laplacian, and
// B[e][m] = -hb (lap phi_m + 2 v_J . grad phi_m + ddjas phi_m) + vloc phi_m.  The nonlocal part
// sum_b phis[e][b] coef[b][m] is added afterwards by one batched GEMM over all walkers.
template <class T>
__device__ void orbital_local_energy(const Sys<T> &s, const View<T> &v, const EvalRes &res, int lane, double *scr) {
  const int N = s.N, B = s.nbasis, M = s.norb;
  double *orbA = scr + (size_t)N * B;
  double *Bm = orbA + (size_t)N * 5 * M;
  for (int e = 0; e < N; e++) {
    warp_basis<T, 5>(s, v.xs + 3 * e, v.phi, lane);
    warp_orbitals<T, 5>(v.phi, s.call, B, M, orbA + (size_t)e * 5 * M, M, lane);
  }
  const double ddjas = (res.d2j + res.vj2) / N, vloc = (res.pe - res.pe_nl) / N;
  for (int i = lane; i < N * M; i += 32) {
    int e = i / M, m = i - e * M;
    const double *o = orbA + (size_t)e * 5 * M + m;
    const double *vj = v.vacc + 3 * e;
    Bm[i] = -HB * (o[4 * M] + 2 * (vj[0] * o[M] + vj[1] * o[2 * M] + vj[2] * o[3 * M]) + ddjas * o[0]) + vloc * o[0];
  }
  __syncwarp();
}

// CSF and orbital-rotation derivatives from the orbitals and the complete B matrix.
template <class T, bool MD>
__device__ void orbital_csf_derivs(const Sys<T> &s, const View<T> &v, double eloc, int lane, double *scr, double *ol,
                                   double *oe) {
  const int N = s.N, B = s.nbasis, M = s.norb, nmax = s.nmax;
  double *orbA = scr + (size_t)N * B;
  double *Bm = orbA + (size_t)N * 5 * M;
  double *Ta = Bm + (size_t)N * M;
  double *dTa = Ta + (size_t)2 * nmax * M;
  double *Qr = dTa + (size_t)2 * nmax * M;
  double *delo = Qr + (size_t)nmax * nmax;
  double eref = 0;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, e0 = sp ? s.nup : 0;
    if (n == 0) continue;
    const double *A = v.ainv + (sp ? s.nup * s.nup : 0);
    double *Ts = Ta + (size_t)sp * nmax * M, *dTs = dTa + (size_t)sp * nmax * M;
    for (int i = lane; i < n * M; i += 32) {
      int k = i / M, m = i - k * M;
      double t = 0, q = 0;
      for (int e = 0; e < n; e++) {
        double a = A[k * n + e];
        t += a * orbA[(size_t)(e0 + e) * 5 * M + m];
        q += a * Bm[(size_t)(e0 + e) * M + m];
      }
      Ts[i] = t;
      dTs[i] = q;
    }
    __syncwarp();
    const int *ro = s.occo[sp];
    double er = 0;
    for (int i = lane; i < n * n; i += 32) {
      int k = i / n, k2 = i - k * n;
      Qr[i] = dTs[k * M + ro[k2]];
      if (k == k2) er += Qr[i];
    }
    eref += warp_sum(er);
    __syncwarp();
    for (int i = lane; i < n * M; i += 32) {
      int k = i / M, m = i - k * M;
      double d = dTs[i];
      for (int k2 = 0; k2 < n; k2++) d -= Qr[k * n + k2] * Ts[k2 * M + m];
      dTs[i] = d;
    }
    __syncwarp();
  }
  if (MD) {
    const int nd0 = s.ndu[0];
    const double *wd = v.wdet;
    for (int sp = 0; sp < 2; sp++) {
      const int n = sp ? s.ndn : s.nup;
      const double *dTs = dTa + (size_t)sp * nmax * M;
      for (int I = lane; I < s.ndu[sp]; I += 32) {
        double a[16], inv[16];
        int k = load_alpha(s, v, sp, I, a);
        double dl = 0;
        if (k) {
          small_det_inv(a, k, inv);
          for (int ia = 0; ia < k; ia++)
            for (int ib = 0; ib < k; ib++)
              dl += inv[ib * k + ia] * dTs[s.dh[sp][4 * I + ia] * M + s.occo[sp][n + s.dpart[sp][4 * I + ib]]];
        }
        delo[(sp ? nd0 : 0) + I] = dl;
      }
    }
    __syncwarp();
    double chi = 0;
    for (int K = lane; K < s.ndet; K += 32) chi += s.ccoef[K] * wd[s.ciu[K]] * wd[nd0 + s.cid[K]];
    chi = warp_sum(chi);
    if (s.norbp > 0) md_orbital_tables(s, v, lane, scr, chi, eref);
    for (int q = 1 + lane; q < s.ncsf; q += 32) {
      double dl = 0, de = 0;
      for (int t = s.csf_off[q]; t < s.csf_off[q + 1]; t++) {
        int K = s.csf_det[t], iu = s.ciu[K], id = s.cid[K];
        double r = wd[iu] * wd[nd0 + id] / chi;
        double eK = eref + delo[iu] + delo[nd0 + id];
        dl += s.csf_cd[t] * r;
        de += s.csf_cd[t] * r * (eK - eloc);
      }
      ol[q - 1] = dl;
      oe[q - 1] = de;
    }
  }
  const int off = MD ? (s.ncsf > 1 ? s.ncsf - 1 : 0) : 0;
  // orbital rotation (i -> j, minus j -> i where both are active): dpsi_orb_bld and
  // deloc_orb_bld (deriv_orb_mod.f90:1486-1629): g = sum_spin (G At)[i][j], h = sum_spin
  // (G B + dG At)[i][j] with G, dG over the spin's orbital set.  One determinant: G = Ainv, so
  // G At = T and G B + dG At = dT.
  const double *GA = MD ? scr + md_ga_offset(s) : Ta, *GH = MD ? GA + (size_t)2 * s.nomax * M : dTa;
  const size_t sps = MD ? (size_t)s.nomax * M : (size_t)nmax * M;
  for (int p = lane; p < s.norbp; p += 32) {
    int4 ij = s.orbp[p];
    double g = 0, h = 0;
    for (int sp = 0; sp < 2; sp++) {
      int oi = s.refpos[sp][ij.x];
      if (oi >= 0) {
        g += GA[sp * sps + (size_t)oi * M + ij.y];
        h += GH[sp * sps + (size_t)oi * M + ij.y];
      }
      int oj = ij.z ? s.refpos[sp][ij.y] : -1;
      if (oj >= 0) {
        g -= GA[sp * sps + (size_t)oj * M + ij.x];
        h -= GH[sp * sps + (size_t)oj * M + ij.x];
      }
    }
    ol[off + p] = g;
    oe[off + p] = h;
  }
  __syncwarp();
}

// part 1: E_L with the Jastrow parameter derivatives and the local part of B; part 2 (after the
// nonlocal part of B was added for all walkers): CSF and orbital-rotation derivatives; part 3: the
// forward pass (E_L, local part of B, tape); part 4: the reverse sweep of the Jastrow parameters.
// One kernel per part, so that each holds only its own code.
template <class T, int NORD, bool MD, int PART>
__global__ void __launch_bounds__(128, 4) k_pgrad(Sys<T> s, State<T> st, Layout L, PGOut out, double r0, double r1,
                                                  double r2, double r3, double r4, double r5, double r6, double r7,
                                                  double r8) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N;
  const int na = J.nct * (J.norda - 1 > 0 ? J.norda - 1 : 0), nb = J.nspin2b * J.nordb;
  const int nt = make_terms(NORD).n, P = na + nb + (NORD > 1 ? J.nct * nt : 0);
  const size_t pgbytes = sizeof(double) * (3 * N + N + 3 * P + N * P + (out.lanesum ? 32 * P : 0));
  const size_t wb = L.base + align16(pgbytes);
  const double R[9] = {r0, r1, r2, r3, r4, r5, r6, r7, r8};
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    char *base = dsm + wb * wib;
    View<T> v = make_view<T>(base, L, st, w, s.N, s.C, s.nbasis, s.nomax, false);
    PGBuf pg;
    double *q = (double *)(base + L.base);
    pg.vt = q; q += 3 * N;
    pg.csum = q; q += N;
    pg.dvn = q; q += P;
    pg.G = q; q += P;
    pg.K = q; q += P;
    pg.old = q; q += N * P;
    pg.dvl = out.lanesum ? q : nullptr;
    pg.P = P; pg.na = na; pg.nb = nb;
    pg.tape = nullptr;
    double *scr = out.scr ? out.scr + (size_t)w * out.scr_stride : nullptr;
    pg.phis = scr;
    if constexpr (PART == 2) {
      orbital_csf_derivs<T, MD>(s, v, out.eloc[w], lane, scr, out.dlnpsi + (size_t)w * out.nfree,
                                out.deloc + (size_t)w * out.nfree);
    } else if constexpr (PART == 4) {
      const int NC = N * s.C, nq = E.nquad;
      // backward pass: one reverse sweep from the tape.  Seeds: -1/2 on every electron's
      // Laplacian of J, -v_e on its gradient, and each nonlocal point's coefficient on the change
      // of J when its electron moves there; the parameter basis functions (every pair, e-n term
      // and point) are recomputed from the positions, in this pass's precision.
      for (int i = lane; i < (int)(pgbytes / sizeof(double)); i += 32) pg.vt[i] = 0.0;
      __syncwarp();
      for (int i = lane; i < 4 * N; i += 32) pg.vt[i] = out.tape_v[(size_t)w * 4 * N + i];  // vt, then csum
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
      if (s.nloc > 0) {
        const int ntask = out.tape_n[w];
        const double *tl = out.tape_nlt + (size_t)w * NC * NLT;
        const double *tc = out.tape_c + (size_t)w * NC * nq;
        for (int t = lane; t < ntask * nq; t += 32) {
          const double coeff = tc[t];
          if (coeff == 0.0) continue;
          const int task = t / nq, q = t - task * nq;
          const double *rec = tl + (size_t)task * NLT;
          const int idx = (int)rec[0], e = idx / s.C, c = idx - e * s.C;
          const double r = rec[1], *cc = s.cent + 3 * c;
          double xn[3];
#pragma unroll
          for (int k = 0; k < 3; k++)
            xn[k] = cc[k] + r * (R[3 * k] * s.quad->q0[q][0] + R[3 * k + 1] * s.quad->q0[q][1] + R[3 * k + 2] * s.quad->q0[q][2]);
          if (pg.dvl) point_param_values<T, NORD, true>(s, J, v, e, xn, coeff, pg, nullptr);
          else point_param_values<T, NORD, false>(s, J, v, e, xn, coeff, pg, nullptr);
        }
        if (pg.dvl) {
          __syncwarp();
          for (int p = lane; p < P; p += 32) {
            double a = 0;
            for (int l = 0; l < 32; l++) a += pg.dvl[p * 32 + l];
            pg.dvn[p] += a;
          }
        }
      }
      __syncwarp();
      jastrow_param_pass<T, NORD>(s, J, v, pg, lane);
      pg_finish<T, NORD>(s, J, pg, out, w, lane, MD);
    } else {
    const int NC = N * s.C, nq = E.nquad;
    for (int i = lane; i < (int)(pgbytes / sizeof(double)); i += 32) pg.vt[i] = 0.0;
    if (scr)
      for (int i = lane; i < N * s.nbasis; i += 32) scr[i] = 0.0;
    for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
    if (PART == 3 && s.nloc > 0) pg.tape = out.tape_c + (size_t)w * NC * nq;
    __syncwarp();
    EvalRes res;
    full_eval<T, NORD, MD, true>(s, J, E, st, w, v, R, lane, false, res, &pg);
    __syncwarp();
    if (scr) orbital_local_energy<T>(s, v, res, lane, scr);
    if (lane == 0) out.eloc[w] = res.eloc;
    if constexpr (PART == 3) {
      // forward pass: the tape for the backward pass
      for (int i = lane; i < 4 * N; i += 32) out.tape_v[(size_t)w * 4 * N + i] = pg.vt[i];
      if (lane == 0) out.tape_n[w] = res.ntask;
      mirror_store(v, st, w, N, s.C, lane);
      __syncwarp();
    } else {
      jastrow_param_pass<T, NORD>(s, J, v, pg, lane);
      pg_finish<T, NORD>(s, J, pg, out, w, lane, MD);
    }
    }
  }
}

// O/H packing: Oa[w] = wt (1, O_w), Mb[w] = (E_L, E_L O_w + dE_w)
static __global__ void k_pack_oh(int W, int P, const double *dl, const double *de, const double *el, const double *wt,
                          double *Oa, double *Ow, double *Mb) {
  const int P1 = P + 1;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)W * P1; i += (size_t)gridDim.x * blockDim.x) {
    int w = (int)(i / P1), p = (int)(i - (size_t)w * P1);
    double o = p ? dl[(size_t)w * P + p - 1] : 1.0;
    double m = p ? el[w] * o + de[(size_t)w * P + p - 1] : el[w];
    double ww = wt ? wt[w] : 1.0;
    Oa[i] = o;
    Ow[i] = ww * o;
    Mb[i] = ww * m;
  }
}
