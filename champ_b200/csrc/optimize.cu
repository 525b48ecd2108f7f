// optimize.cu -- the optimisation driver's checks and its choice of the stabilisation constant
// (host code): which linear-method steps the reference rejects (wf_update_and_check,
// qmc/optimization_mod.f90:1730-1840), the correlated-sampling energies of a trial step on the
// current walkers, and one stabilised linear-method iteration (adjust_diag_stab and
// wf_update_and_check_and_stab, qmc/optimization_mod.f90:1845-2250, with the parabolic fit of
// qmc/vmc/quad_min.f90).
//
// The reference samples its three trial wave functions with an extra short VMC run (nwf = 3,
// correlated sampling).  Here the walkers the context holds -- sampled from the current wave
// function -- are reweighted to each trial wave function by w = (psi_new / psi_old)^2, which needs
// one full evaluation per trial and no sampling.  The reference ignores a correlated run whose
// autocorrelation time exceeds 50; the walkers here are independent, so the same role is played by
// the weights' effective sample size: a trial whose (sum w)^2 / sum w^2 is below 1/50 of the
// walkers is not reliable.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/champ_b200.h"
#include "ctx.h"

int champ_fail(int code, const std::string &msg);

namespace {

// Energy, its statistical error and sigma of the current walkers reweighted by exp(2 dlnpsi).
struct CorrEnergy {
  double e = 0, err = 0, sigma = 0, ess = 0;
  bool finite = true;
};

CorrEnergy weighted(const std::vector<double> &el, const std::vector<double> *dl) {
  CorrEnergy r;
  const size_t W = el.size();
  double lmax = 0;
  if (dl)
    for (size_t i = 0; i < W; i++) lmax = std::max(lmax, 2 * (*dl)[i]);
  std::vector<double> w(W, 1.0);
  double sw = 0, sw2 = 0, swe = 0;
  for (size_t i = 0; i < W; i++) {
    if (dl) w[i] = std::exp(2 * (*dl)[i] - lmax);
    if (!std::isfinite(w[i]) || !std::isfinite(el[i])) { r.finite = false; return r; }
    sw += w[i];
    sw2 += w[i] * w[i];
    swe += w[i] * el[i];
  }
  r.e = swe / sw;
  double v = 0, v2 = 0;
  for (size_t i = 0; i < W; i++) {
    const double d = el[i] - r.e;
    v += w[i] * d * d;
    v2 += w[i] * w[i] * d * d;
  }
  r.sigma = std::sqrt(v / sw);
  r.err = std::sqrt(v2) / sw;
  r.ess = sw * sw / sw2;
  return r;
}

int eval_current(champ_ctx *c, std::vector<double> &el, std::vector<double> &lnpsi) {
  el.assign(c->W, 0.0);
  lnpsi.assign(c->W, 0.0);
  champ_eval_out o{};
  o.energy = el.data();
  o.lnpsi = lnpsi.data();
  return champ_eval_full(c, &o);
}

}  // namespace

extern "C" {

int champ_check_param_step(const champ_ctx *c, const double *dp, double psi_lin_var_norm, int32_t *bad) {
  if (!c || !dp || !bad) return champ_fail(CHAMP_EINVAL, "null argument");
  const Params &q = c->par;
  const int ncsf = c->ncsfp, norb = c->norbp, nj = c->nparm_jas, P = c->nfree;
  int r = 0;
  // root-mean-square variation over the parameters of a group that the step changes (the
  // reference divides by the number of optimised parameters)
  auto norm = [&](int k0, int n) {
    double s = 0;
    int m = 0;
    for (int k = k0; k < k0 + n; k++) {
      s += dp[k] * dp[k];
      m += dp[k] != 0.0;
    }
    return m ? std::sqrt(s / m) : 0.0;
  };
  for (int k = 0; k < P; k++)
    if (!std::isfinite(dp[k])) { *bad = 2; return CHAMP_OK; }
  // norm of the CSF coefficient variations; of the Jastrow variations (3-dimensional systems)
  if (ncsf && norm(0, ncsf) > 1.0) r = 1;
  if (nj && norm(ncsf + norb, nj) > std::max(10.0, 5.0 / q.scalek)) r = 1;
  // the Pade denominator parameter b2 of every spin set after the step (a2 is not optimised)
  const int jb = ncsf + norb + c->nct * std::max(0, q.norda - 1);
  const double parm2min = -q.scalek, amax_nonlin = 100.0;
  for (int is = 0; is < q.nspin2b; is++) {
    const double b2 = q.b[(size_t)is * (q.nordb + 1) + 1] + (q.nordb >= 1 ? dp[jb + is * q.nordb] : 0.0);
    if (b2 > amax_nonlin) r = std::max(r, 1);
    if (b2 < parm2min) r = 2;
  }
  for (int it = 0; it < c->nct; it++) {
    const double a2 = q.a4[(size_t)it * (q.norda + 1) + 1];
    if (a2 > amax_nonlin) r = std::max(r, 1);
    if (a2 < parm2min) r = 2;
  }
  // total parameter variation and the linear wave-function variation
  if (norm(0, P) > 10.0) r = std::max(r, 1);
  if (psi_lin_var_norm > 10.0) r = std::max(r, 1);
  *bad = r;
  return CHAMP_OK;
}

int champ_eval_param_step(champ_ctx *c, const double *dp, double *eloc, double *dlnpsi) {
  if (!c || !dp) return champ_fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return champ_fail(CHAMP_ESTATE, "no walkers set");
  std::vector<double> e0, l0, e1, l1;
  int rc = eval_current(c, e0, l0);
  if (rc) return rc;
  const Params saved = c->par;
  rc = champ_apply_param_step(c, dp);
  if (!rc) rc = eval_current(c, e1, l1);
  c->par = saved;  // back to the current wave function, also after a failed evaluation
  const int rc2 = champ_set_params(c, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  if (rc2) return rc2;
  for (int i = 0; i < c->W; i++) {
    if (eloc) eloc[i] = e1[i];
    if (dlnpsi) dlnpsi[i] = l1[i] - l0[i];
  }
  return CHAMP_OK;
}

int champ_linear_method_step(champ_ctx *c, int32_t nsel, const int32_t *sel, const double *S, const double *H,
                             double sigma, double p_var, double *diag_stab, double *dp_out, double *info) {
  if (!c || !S || !H || !diag_stab) return champ_fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return champ_fail(CHAMP_ESTATE, "no walkers set");
  if (p_var < 0 || p_var > 1) return champ_fail(CHAMP_EINVAL, "p_var must lie in [0, 1]");
  const int P = c->nfree;
  if (!sel) nsel = P;
  if (nsel < 1 || nsel > P) return champ_fail(CHAMP_EINVAL, "bad parameter selection");
  std::vector<int> idx(nsel);
  int ncsf_sel = 0;
  for (int i = 0; i < nsel; i++) {
    idx[i] = sel ? sel[i] : i;
    if (idx[i] < 0 || idx[i] >= P || (i && idx[i] <= idx[i - 1]))
      return champ_fail(CHAMP_EINVAL, "parameter selection must be increasing indices below P");
    if (idx[i] < c->ncsfp) ncsf_sel++;
  }
  const double add_diag_max = 1e10;

  // the step for one stabilisation constant, scattered into the full parameter vector
  std::vector<double> dsel(nsel);
  auto solve = [&](double stab, std::vector<double> &full, double *inf4, int32_t *bad) -> int {
    double inf[4] = {0, 0, 0, 0};
    int rc = champ_linear_update(nsel, ncsf_sel, S, H, sigma, stab, 0, dsel.data(), inf);
    if (rc) return rc;
    full.assign(P, 0.0);
    for (int i = 0; i < nsel; i++) full[idx[i]] = dsel[i];
    if (inf4) std::copy(inf, inf + 4, inf4);
    return champ_check_param_step(c, full.data(), inf[2], bad);
  };

  // the current wave function's energy on these walkers
  std::vector<double> el, lnpsi;
  int rc = eval_current(c, el, lnpsi);
  if (rc) return rc;
  const CorrEnergy cur = weighted(el, nullptr);
  const double ene_var_sav = (1 - p_var) * cur.e + p_var * cur.sigma * cur.sigma;
  const double W = (double)c->W;

  double add1 = *diag_stab;
  int loops = 0;
  CorrEnergy ce[3];
  double add[3];
  for (;; loops++) {
    if (loops >= 15) return champ_fail(CHAMP_EINVAL, "linear method: stabilisation increased 15 times, steps still bad");
    if (add1 >= add_diag_max) return champ_fail(CHAMP_EINVAL, "linear method: diag_stab too large");
    add[0] = add1;
    add[1] = 0.1 * add1;
    add[2] = 10 * add1;
    int32_t bad[3];
    std::vector<double> full[3];
    for (int k = 0; k < 3; k++) {
      rc = solve(add[k], full[k], nullptr, &bad[k]);
      if (rc) return rc;
    }
    if (bad[0] || bad[1] || bad[2]) {
      add1 *= std::pow(10.0, std::min(bad[0] + bad[1] + bad[2], 3));
      continue;
    }
    std::vector<double> e(c->W), d(c->W);
    for (int k = 0; k < 3; k++) {
      rc = champ_eval_param_step(c, full[k].data(), e.data(), d.data());
      if (rc) return rc;
      ce[k] = weighted(e, &d);
    }
    if (!ce[0].finite || ce[0].ess < W / 50) {  // the central trial is not reliable
      add1 *= 10;
      continue;
    }
    auto worse = [&](const CorrEnergy &x) {
      return !x.finite || x.sigma > (2.5 - p_var) * cur.sigma ||
             x.e - cur.e > 3 * (1 + p_var) * std::sqrt(x.err * x.err + cur.err * cur.err);
    };
    if ((worse(ce[0]) && worse(ce[1]) && worse(ce[2])) || !ce[2].finite) {
      add1 *= 1000;
      continue;
    }
    break;
  }

  // the stabilisation constant: parabolic fit of the objective in log10(add_diag) (quad_min)
  int nrel = 0;
  for (int k = 0; k < 3; k++) nrel += (ce[k].finite && ce[k].ess >= W / 50);
  double ev[3], lg[3];
  for (int k = 0; k < 3; k++) {
    ev[k] = (1 - p_var) * ce[k].e + p_var * ce[k].sigma * ce[k].sigma;
    lg[k] = std::log10(add[k]);
  }
  double lmin;
  if (nrel == 3) {
    // the parabola through the three points: ev = b0 + b1 t + b2 t^2 with t = lg - lg[0]
    const double t1 = lg[1] - lg[0], t2 = lg[2] - lg[0];
    const double s1 = (ev[1] - ev[0]) / t1, s2 = (ev[2] - ev[0]) / t2;
    const double b2 = (s2 - s1) / (t2 - t1), b1 = s1 - b2 * t1;
    if (b2 > 0) {
      lmin = lg[0] - 0.5 * b1 / b2;
      lmin = std::min(std::max(lmin, lg[0] - 2), lg[0] + 2);
    } else {
      int kb = 0;
      for (int k = 1; k < 3; k++)
        if (ev[k] + (1 - p_var) * 3 * ce[k].err < ev[kb] + (1 - p_var) * 3 * ce[kb].err) kb = k;
      lmin = lg[kb];
    }
    // conservative choices when the smaller constants have clearly larger errors
    if (lmin < lg[0] && ce[1].err > 1.1 * ce[0].err) lmin = lg[0];
    if (lmin < lg[2] && ce[0].err > 1.1 * ce[2].err && ce[1].err > 1.1 * ce[2].err) lmin = lg[2];
    lmin = std::max(lmin, -12.0);
  } else {
    lmin = lg[0];
    if (ev[0] > ene_var_sav) lmin += 1;
  }
  double stab = std::min(std::pow(10.0, lmin), add_diag_max);

  // the update with that constant, made larger until the step passes the checks
  std::vector<double> full;
  double inf4[4];
  for (int loop = 0;; loop++) {
    if (loop >= 50) return champ_fail(CHAMP_EINVAL, "linear method: step still rejected after 50 increases");
    int32_t bad;
    rc = solve(stab, full, inf4, &bad);
    if (rc) return rc;
    if (!bad) break;
    stab = std::min(stab * 10, add_diag_max);
    if (stab >= add_diag_max) return champ_fail(CHAMP_EINVAL, "linear method: diag_stab too large");
  }
  rc = champ_apply_param_step(c, full.data());
  if (rc) return rc;
  *diag_stab = stab;
  if (dp_out) std::copy(full.begin(), full.end(), dp_out);
  if (info) {
    info[0] = inf4[0];  // selected eigenvalue
    info[1] = inf4[2];  // wave-function variation of the selection
    info[2] = cur.e;    // energy of the walkers before the step
    info[3] = cur.err;
    for (int k = 0; k < 3; k++) info[4 + k] = ce[k].e;  // correlated energies of add_diag(1..3)
    info[7] = (double)loops;
  }
  return CHAMP_OK;
}

}  // extern "C"
