// linear.cu -- the linear method's parameter update from the accumulated O/H sums (host code).
//
// From the sums champ_accumulate_oh returns, S = sum_w wt (1,O)(1,O)^T and
// H = sum_w wt (1,O)(E_L, E_L O + dE_L)^T, builds the overlap and Hamiltonian matrices of the
// current wave function and its first-order parameter derivatives (ovlp_lin_bld and
// ham_lin_energy_bld, qmc/opt_lin_mod.f90:249-555), renormalises them by the overlap's diagonal
// (ovlp_lin_renorm_bld, :350), adds the 'identity' stabilisation to the Hamiltonian's diagonal
// (ham_lin_renorm_stab_bld, :756), solves the generalised non-symmetric eigenproblem H c = E S c
// (the reference calls LAPACK dggev, :885), selects the eigenvector as delta_lin_bld does
// (:820-1265: the lowest eigenvalue inside the energy window unless its wave-function variation
// is 100 times that of the smallest one) and returns the parameter variations with the
// semi-orthogonal normalisation of the nonlinear parameters (xi = 1).
//
// The eigenproblem: S = L L^T (Cholesky), M = L^-1 H L^-T, M reduced to Hessenberg form by
// Householder reflections, then to complex Schur form T = Z^H M Z by shifted QR sweeps (Givens
// rotations, Wilkinson shifts), eigenvectors of T by back substitution, c = L^-T Z y.
#include <algorithm>
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "../../include/champ_b200.h"

int champ_fail(int code, const std::string &msg);

namespace {

using cd = std::complex<double>;

// Eigenvalues and right eigenvectors of a real n x n matrix A (row-major).  V column k is the
// eigenvector of lam[k].  Returns false if the QR sweeps do not converge.
bool eig_real(int n, const std::vector<double> &A, std::vector<cd> &lam, std::vector<cd> &V) {
  std::vector<double> Hm(A), Q((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) Q[(size_t)i * n + i] = 1.0;
  std::vector<double> v(n);
  for (int k = 0; k + 2 < n; k++) {
    const int m = n - k - 1;
    double alpha = 0;
    for (int i = 0; i < m; i++) alpha += Hm[(size_t)(k + 1 + i) * n + k] * Hm[(size_t)(k + 1 + i) * n + k];
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    if (Hm[(size_t)(k + 1) * n + k] > 0) alpha = -alpha;
    double vn = 0;
    for (int i = 0; i < m; i++) {
      v[i] = Hm[(size_t)(k + 1 + i) * n + k] - (i == 0 ? alpha : 0.0);
      vn += v[i] * v[i];
    }
    if (vn == 0.0) continue;
    for (int j = k; j < n; j++) {  // rows k+1.. of H
      double s = 0;
      for (int i = 0; i < m; i++) s += v[i] * Hm[(size_t)(k + 1 + i) * n + j];
      const double f = 2 * s / vn;
      for (int i = 0; i < m; i++) Hm[(size_t)(k + 1 + i) * n + j] -= f * v[i];
    }
    for (int i = 0; i < n; i++) {  // columns k+1.. of H and of Q
      double s = 0, t = 0;
      for (int j = 0; j < m; j++) {
        s += Hm[(size_t)i * n + k + 1 + j] * v[j];
        t += Q[(size_t)i * n + k + 1 + j] * v[j];
      }
      const double f = 2 * s / vn, g = 2 * t / vn;
      for (int j = 0; j < m; j++) {
        Hm[(size_t)i * n + k + 1 + j] -= f * v[j];
        Q[(size_t)i * n + k + 1 + j] -= g * v[j];
      }
    }
    for (int i = k + 2; i < n; i++) Hm[(size_t)i * n + k] = 0.0;
  }
  std::vector<cd> T(Hm.begin(), Hm.end()), Z(Q.begin(), Q.end());
  auto t = [&](int i, int j) -> cd & { return T[(size_t)i * n + j]; };
  double tnorm = 0;
  for (const cd &x : T) tnorm = std::max(tnorm, std::abs(x));
  const double eps = 2.220446049250313e-16;
  std::vector<cd> cs(n), sn(n);
  int hi = n - 1, iter = 0, total = 0;
  while (hi >= 1) {
    int l = hi;
    for (; l > 0; l--) {
      double sc = std::abs(t(l - 1, l - 1)) + std::abs(t(l, l));
      if (sc == 0.0) sc = tnorm;
      if (std::abs(t(l, l - 1)) <= eps * sc || std::abs(t(l, l - 1)) <= 1e-3 * eps * tnorm) {
        t(l, l - 1) = 0.0;
        break;
      }
    }
    if (l == hi) {
      hi--;
      iter = 0;
      continue;
    }
    if (++iter > 200 || ++total > 100 * n + 1000) return false;
    const cd a = t(hi - 1, hi - 1), b = t(hi - 1, hi), c = t(hi, hi - 1), d = t(hi, hi);
    const cd disc = std::sqrt(0.25 * (a - d) * (a - d) + b * c);
    const cd m1 = 0.5 * (a + d) + disc, m2 = 0.5 * (a + d) - disc;
    cd mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
    if (iter % 10 == 0) mu = d + std::abs(t(hi, hi - 1));  // exceptional shift
    for (int i = l; i <= hi; i++) t(i, i) -= mu;
    for (int k = l; k < hi; k++) {
      const cd x = t(k, k), y = t(k + 1, k);
      const double r = std::sqrt(std::norm(x) + std::norm(y));
      cd ck = 1.0, sk = 0.0;
      if (r > 0) { ck = x / r; sk = y / r; }
      cs[k] = ck;
      sn[k] = sk;
      for (int j = k; j < n; j++) {
        const cd t1 = t(k, j), t2 = t(k + 1, j);
        t(k, j) = std::conj(ck) * t1 + std::conj(sk) * t2;
        t(k + 1, j) = -sk * t1 + ck * t2;
      }
    }
    for (int k = l; k < hi; k++) {
      const cd ck = cs[k], sk = sn[k];
      const int r1 = std::min(k + 2, hi);
      for (int i = 0; i <= r1; i++) {
        const cd t1 = t(i, k), t2 = t(i, k + 1);
        t(i, k) = t1 * ck + t2 * sk;
        t(i, k + 1) = -t1 * std::conj(sk) + t2 * std::conj(ck);
      }
      for (int i = 0; i < n; i++) {
        cd &z1 = Z[(size_t)i * n + k], &z2 = Z[(size_t)i * n + k + 1];
        const cd t1 = z1, t2 = z2;
        z1 = t1 * ck + t2 * sk;
        z2 = -t1 * std::conj(sk) + t2 * std::conj(ck);
      }
    }
    for (int i = l; i <= hi; i++) t(i, i) += mu;
  }
  lam.resize(n);
  for (int i = 0; i < n; i++) lam[i] = t(i, i);
  V.assign((size_t)n * n, 0.0);
  std::vector<cd> y(n);
  const double small = std::max(eps * tnorm, 1e-300);
  for (int k = 0; k < n; k++) {
    std::fill(y.begin(), y.end(), cd(0.0));
    y[k] = 1.0;
    for (int i = k - 1; i >= 0; i--) {
      cd s = 0;
      for (int j = i + 1; j <= k; j++) s += t(i, j) * y[j];
      cd den = t(i, i) - lam[k];
      if (std::abs(den) < small) den = small;
      y[i] = -s / den;
    }
    double nrm = 0;
    for (int i = 0; i < n; i++) {
      cd acc = 0;
      for (int j = 0; j <= k; j++) acc += Z[(size_t)i * n + j] * y[j];
      V[(size_t)i * n + k] = acc;
      nrm += std::norm(acc);
    }
    nrm = std::sqrt(nrm);
    if (nrm > 0)
      for (int i = 0; i < n; i++) V[(size_t)i * n + k] /= nrm;
  }
  return true;
}

}  // namespace

extern "C" int champ_linear_update(int32_t nparm, int32_t ncsf, const double *S, const double *H, double sigma,
                                   double diag_stab, int32_t select, double *dp, double *info) {
  if (nparm < 1 || ncsf < 0 || ncsf > nparm || !S || !H || !dp) return champ_fail(CHAMP_EINVAL, "linear update: bad argument");
  const int P = nparm, n1 = P + 1;
  for (size_t i = 0; i < (size_t)n1 * n1; i++)
    if (!std::isfinite(S[i]) || !std::isfinite(H[i]))
      return champ_fail(CHAMP_EINVAL, "linear update: non-finite entries in S or H (a walker with a non-finite E_L "
                                      "or derivative entered the sums)");
  const double W = S[0];
  if (!(W > 0)) return champ_fail(CHAMP_EINVAL, "linear update: the summed weight S[0][0] must be positive");
  auto s = [&](int a, int b) { return S[(size_t)a * n1 + b] / W; };
  auto h = [&](int a, int b) { return H[(size_t)a * n1 + b] / W; };
  const double el = h(0, 0);
  std::vector<double> o(P), oe(P), dl(P);  // <O_i>, <O_i E_L>, <dE_L_i>
  for (int i = 0; i < P; i++) {
    o[i] = s(0, i + 1);
    oe[i] = h(i + 1, 0);
    dl[i] = h(0, i + 1) - h(i + 1, 0);
  }
  // parameters without variance (a zero derivative on every sample) take no step
  std::vector<int> act;
  double dmax = 0;
  for (int i = 0; i < P; i++) dmax = std::max(dmax, s(i + 1, i + 1) - o[i] * o[i]);
  for (int i = 0; i < P; i++)
    if (s(i + 1, i + 1) - o[i] * o[i] > 1e-14 * dmax) act.push_back(i);
  const int na = (int)act.size(), n = na + 1;
  for (int i = 0; i < P; i++) dp[i] = 0.0;
  if (na == 0) return champ_fail(CHAMP_EINVAL, "linear update: no parameter has a non-zero variance");
  // overlap and Hamiltonian of psi and its derivatives (index 0: psi), renormalised
  std::vector<double> ov((size_t)n * n, 0.0), hm((size_t)n * n, 0.0), rn(n, 1.0);
  ov[0] = 1.0;
  hm[0] = el;
  for (int a = 0; a < na; a++) {
    const int i = act[a];
    hm[(size_t)(a + 1) * n] = oe[i] - o[i] * el;
    hm[a + 1] = oe[i] - o[i] * el + dl[i];
    for (int b = 0; b < na; b++) {
      const int j = act[b];
      ov[(size_t)(a + 1) * n + b + 1] = s(i + 1, j + 1) - o[i] * o[j];
      hm[(size_t)(a + 1) * n + b + 1] = h(i + 1, j + 1) - o[i] * dl[j] - o[j] * oe[i] - o[i] * oe[j] + o[i] * o[j] * el;
    }
  }
  for (int a = 1; a < n; a++) rn[a] = std::sqrt(ov[(size_t)a * n + a]);
  std::vector<double> ovr(ov), hmr(hm);
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++) {
      ovr[(size_t)a * n + b] /= rn[a] * rn[b];
      hmr[(size_t)a * n + b] /= rn[a] * rn[b];
    }
  for (int a = 1; a < n; a++) hmr[(size_t)a * n + a] += diag_stab;
  // S = L L^T
  std::vector<double> L((size_t)n * n, 0.0);
  double shift = 0;
  for (int attempt = 0; attempt < 8; attempt++) {
    bool ok = true;
    for (int j = 0; j < n && ok; j++) {
      double d = ovr[(size_t)j * n + j] + shift;
      for (int k = 0; k < j; k++) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
      if (!(d > 0)) { ok = false; break; }
      L[(size_t)j * n + j] = std::sqrt(d);
      for (int i = j + 1; i < n; i++) {
        double x = ovr[(size_t)i * n + j];
        for (int k = 0; k < j; k++) x -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
        L[(size_t)i * n + j] = x / L[(size_t)j * n + j];
      }
    }
    if (ok) break;
    if (attempt == 7) return champ_fail(CHAMP_EINVAL, "linear update: the overlap matrix is not positive definite");
    shift = shift == 0 ? 1e-12 : shift * 100;
  }
  // M = L^-1 H L^-T: X = L^-1 H (columns), M^T = L^-1 X^T
  std::vector<double> X(hmr), M((size_t)n * n);
  for (int c = 0; c < n; c++)
    for (int i = 0; i < n; i++) {
      double x = X[(size_t)i * n + c];
      for (int k = 0; k < i; k++) x -= L[(size_t)i * n + k] * X[(size_t)k * n + c];
      X[(size_t)i * n + c] = x / L[(size_t)i * n + i];
    }
  for (int r = 0; r < n; r++)
    for (int i = 0; i < n; i++) {  // M[r][i] = (L^-1 X^T)[i][r]
      double x = X[(size_t)r * n + i];
      for (int k = 0; k < i; k++) x -= L[(size_t)i * n + k] * M[(size_t)r * n + k];
      M[(size_t)r * n + i] = x / L[(size_t)i * n + i];
    }
  std::vector<cd> lam, Y;
  if (!eig_real(n, M, lam, Y)) return champ_fail(CHAMP_ECUDA, "linear update: eigenvalue iteration did not converge");
  // c = L^-T y for every eigenvector (renormalised basis); real parts as the reference uses them
  std::vector<double> C((size_t)n * n);
  std::vector<cd> cv(n);
  for (int k = 0; k < n; k++) {
    for (int i = n - 1; i >= 0; i--) {
      cd x = Y[(size_t)i * n + k];
      for (int j = i + 1; j < n; j++) x -= L[(size_t)j * n + i] * cv[j];
      cv[i] = x / L[(size_t)i * n + i];
    }
    for (int i = 0; i < n; i++) C[(size_t)i * n + k] = cv[i].real();
  }
  // wave-function variation of the non-CSF parameters per eigenvector (first component set to 1)
  auto varnorm = [&](int k) {
    double v = 0;
    for (int a = 0; a < na; a++) {
      if (act[a] < ncsf) continue;
      for (int b = 0; b < na; b++) {
        if (act[b] < ncsf) continue;
        v += C[(size_t)(a + 1) * n + k] * C[(size_t)(b + 1) * n + k] * ovr[(size_t)(a + 1) * n + b + 1];
      }
    }
    const double c0 = C[k];
    return c0 != 0 ? v / (c0 * c0) : 1e300;
  };
  // eigenvalues of complex-conjugate pairs are left out of the choice: their eigenvectors have no
  // real representative (the real part depends on an arbitrary phase)
  std::vector<char> real_k(n, 1);
  int nreal = 0;
  for (int k = 0; k < n; k++) {
    real_k[k] = std::fabs(lam[k].imag()) <= 1e-8 * std::max(1.0, std::abs(lam[k]));
    nreal += real_k[k];
  }
  if (nreal == 0) std::fill(real_k.begin(), real_k.end(), 1);
  int ksmall = -1, klow = -1, kfirst = -1;
  double smallest = 9e99, lowest = 9e99, lowest_all = 9e99;
  const double upper = el + 0.01, lower = sigma > 0 ? el - sigma : -9e99;
  for (int k = 0; k < n; k++) {
    if (!real_k[k]) continue;
    if (ksmall < 0) ksmall = kfirst = k;
    const double e = lam[k].real(), nv = varnorm(k);
    lowest_all = std::min(lowest_all, e);
    if (nv >= 0 && (nv < smallest || (nv == smallest && e < lam[ksmall].real()))) { smallest = nv; ksmall = k; }
    if (e < upper && e > lower && (e < lowest || (e == lowest && std::fabs(C[k]) > std::fabs(C[klow])))) {
      lowest = e;
      klow = k;
    }
    if (std::fabs(C[k]) > std::fabs(C[kfirst]) || (std::fabs(C[k]) == std::fabs(C[kfirst]) && e < lam[kfirst].real()))
      kfirst = k;
  }
  int ksel;
  if (select == 1 && klow >= 0) ksel = klow;
  else if (select == 2) ksel = kfirst;
  else if (select == 3 || (select == 1 && klow < 0)) ksel = ksmall;
  else ksel = (klow >= 0 && varnorm(klow) < 100 * smallest) ? klow : ksmall;
  // back to the parameters' own scale, first component 1, semi-orthogonal normalisation
  std::vector<double> c(n);
  for (int a = 0; a < n; a++) c[a] = C[(size_t)a * n + ksel] / rn[a];
  const double c0 = c[0];
  if (c0 == 0) return champ_fail(CHAMP_EINVAL, "linear update: the selected eigenvector has no component on psi");
  for (int a = 0; a < n; a++) c[a] /= c0;
  double first = 1.0, vnorm = 0;
  for (int a = 0; a < na; a++)
    if (act[a] < ncsf) first -= c[a + 1] * o[act[a]];
  for (int a = 0; a < na; a++)
    for (int b = 0; b < na; b++)
      if (act[a] >= ncsf && act[b] >= ncsf) vnorm += c[a + 1] * c[b + 1] * ov[(size_t)(a + 1) * n + b + 1];
  for (int a = 0; a < na; a++) dp[act[a]] = c[a + 1] / first;
  if (info) {
    info[0] = lam[ksel].real();
    info[1] = lowest_all;
    info[2] = vnorm;
    info[3] = (double)na;
  }
  return CHAMP_OK;
}
