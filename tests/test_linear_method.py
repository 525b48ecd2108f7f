"""champ_linear_update (host code of the engine library) against a NumPy/SciPy restatement of the
linear method's update (qmc/opt_lin_mod.f90: ovlp_lin_bld, ham_lin_energy_bld, renormalisation,
'identity' stabilisation, dggev, delta_lin_bld's default eigenvector choice and semi-orthogonal
normalisation).  CPU only: the update needs no GPU."""
import numpy as np
import pytest
import scipy.linalg

from champ_b200.engine import linear_update


def sums(O, E, dE, wt):
    """The O/H sums of champ_accumulate_oh: S = sum wt (1,O)(1,O)^T, H = sum wt (1,O)(E, E O + dE)^T."""
    W = len(E)
    Oa = np.hstack([np.ones((W, 1)), O])
    Mb = np.hstack([E[:, None], E[:, None] * O + dE])
    return (Oa * wt[:, None]).T @ Oa, (Oa * wt[:, None]).T @ Mb


def reference_update(S, H, ncsf, sigma, stab):
    W = S[0, 0]
    s, h = S / W, H / W
    P = S.shape[0] - 1
    o, oe, el = s[0, 1:], h[1:, 0], h[0, 0]
    dl = h[0, 1:] - h[1:, 0]
    ov = np.zeros((P + 1, P + 1))
    hm = np.zeros((P + 1, P + 1))
    ov[0, 0] = 1
    ov[1:, 1:] = s[1:, 1:] - np.outer(o, o)
    hm[0, 0] = el
    hm[1:, 0] = oe - o * el
    hm[0, 1:] = oe - o * el + dl
    hm[1:, 1:] = h[1:, 1:] - np.outer(o, dl) - np.outer(oe, o) - np.outer(o, oe) + np.outer(o, o) * el
    rn = np.sqrt(np.diag(ov))
    ovr, hmr = ov / np.outer(rn, rn), hm / np.outer(rn, rn)
    hmr[1:, 1:] += stab * np.eye(P)
    lam, C = scipy.linalg.eig(hmr, ovr)
    lam, C = lam.real, C.real

    def vnorm(k):
        c = C[:, k]
        m = np.arange(1, P + 1) > ncsf
        return (c[1:][m[1 - 1:]] @ ovr[1:, 1:][np.ix_(m, m)] @ c[1:][m]) / c[0] ** 2 if c[0] != 0 else 1e300

    lam_c = scipy.linalg.eigvals(hmr, ovr)
    real = np.abs(lam_c.imag) <= 1e-8 * np.maximum(1.0, np.abs(lam_c))  # complex pairs are not chosen
    norms = np.array([vnorm(k) for k in range(P + 1)])
    ok = (norms >= 0) & real
    ksmall = int(np.argmin(np.where(ok, norms, np.inf)))
    win = (lam < el + 0.01) & (lam > (el - sigma if sigma > 0 else -np.inf)) & real
    klow = int(np.argmin(np.where(win, lam, np.inf))) if win.any() else -1
    k = klow if (klow >= 0 and norms[klow] < 100 * norms[ksmall]) else ksmall
    c = C[:, k] / rn
    c = c / c[0]
    first = 1 - np.dot(c[1:ncsf + 1], o[:ncsf])
    return c[1:] / first, lam[k]


@pytest.mark.parametrize("P,ncsf,stab,seed", [(6, 0, 0.0, 1), (12, 3, 0.1, 2), (40, 5, 0.01, 3), (90, 0, 1.0, 4)])
def test_linear_update_matches_scipy(P, ncsf, stab, seed):
    rng = np.random.default_rng(seed)
    W = 4000
    O = rng.standard_normal((W, P)) @ rng.standard_normal((P, P)) * 0.3
    E = -10 + 0.5 * rng.standard_normal(W) + O @ rng.normal(0, 0.05, P)
    dE = 0.2 * rng.standard_normal((W, P)) + 0.1 * O * E[:, None] / 10
    wt = rng.uniform(0.5, 1.5, W)
    S, H = sums(O, E, dE, wt)
    sigma = np.sqrt(np.average((E - np.average(E, weights=wt)) ** 2, weights=wt))
    dp, info = linear_update(S, H, ncsf=ncsf, sigma=sigma, diag_stab=stab)
    ref, lam = reference_update(S, H, ncsf, sigma, stab)
    assert abs(info[0] - lam) <= 1e-9 * max(1, abs(lam))
    assert np.allclose(dp, ref, rtol=1e-7, atol=1e-9 * np.abs(ref).max()), np.abs(dp - ref).max()


def test_linear_update_recovers_a_linear_parameter():
    """psi(p) linear in p with an exactly known optimum: for E_L samples from H psi = E psi in a
    two-function basis the eigenvector gives the variation to the lower eigenstate."""
    rng = np.random.default_rng(7)
    W = 20000
    # a two-state model: O = phi1/phi0 samples, E_L of psi0 with a coupling
    O = rng.standard_normal((W, 1))
    E = -1.0 + 0.3 * O[:, 0] + 0.01 * rng.standard_normal(W)
    dE = 0.3 * O * 0 + 0.5 * O - 0.3 * O ** 2 * 0
    S, H = sums(O, E, dE, np.ones(W))
    dp, info = linear_update(S, H)
    ref, lam = reference_update(S, H, 0, 0.0, 0.0)
    assert np.allclose(dp, ref, rtol=1e-8)
    assert info[0] <= S[0, 0] and np.isfinite(dp).all()


def test_zero_variance_parameter_takes_no_step():
    rng = np.random.default_rng(9)
    W, P = 3000, 5
    O = rng.standard_normal((W, P))
    O[:, 2] = 0.0
    E = -5 + rng.standard_normal(W)
    dE = 0.1 * rng.standard_normal((W, P))
    dE[:, 2] = 0.0
    S, H = sums(O, E, dE, np.ones(W))
    dp, info = linear_update(S, H, diag_stab=0.1)
    assert dp[2] == 0.0 and info[3] == P - 1
    keep = [0, 1, 3, 4]
    ref, _ = reference_update(S[np.ix_([0] + [k + 1 for k in keep], [0] + [k + 1 for k in keep])],
                              H[np.ix_([0] + [k + 1 for k in keep], [0] + [k + 1 for k in keep])], 0, 0.0, 0.1)
    assert np.allclose(dp[keep], ref, rtol=1e-7)
