"""The reference's C2 pseudopotential example through the oracle (CPU only).

examples/c2_bfd_vtz_rhf_vmc_new.inp runs two carbon pseudo-atoms with 68 basis functions built
on 9 numerical radial functions (examples/basis.1, interpolated by splfit_bas), the BFD
pseudopotential of examples/pseudopot1 (local p channel, nonlocal s channel) with the 6-point
quadrature, and an ijas=4 Jastrow whose e-n, e-e and e-e-n (order 5) coefficients the transcript
prints for every VMC run of its linear-method optimisation.  The fixture tests/golden/c2_bfd.npz
is made from those files by tests/golden/make_c2_bfd_fixture.py.  These tests pin the oracle's
numerical basis, pseudopotential, quadrature and e-e-n Jastrow to the transcript's energies.
"""
import numpy as np
import pytest

from champ_b200 import system as S


@pytest.fixture(scope="module")
def fx():
    return S.c2_bfd_fixture()


def test_fixture_contents(fx):
    meta, coef, gx, gv = fx
    assert coef.shape == (68, 68) and gv.shape == (9, 2000) and gx.shape == (2000,)
    assert meta["nquad"] == 6 and meta["nloc"] == 6 and meta["lpotp1"] == [2]
    runs = meta["runs"]
    assert len(runs) == 11
    assert runs[0]["energy"] == -10.7748993 and runs[0]["energy_err"] == 0.0124482
    assert runs[-1]["energy"] == -11.0176327 and runs[-1]["passes"] == 1233100.0
    assert all(len(r["params"]["c"]) == 23 for r in runs)


def test_numerical_radial_function_interpolates_the_grid(oracle_mod, fx):
    """A cubic spline passes through its knots: the s function of radial table 1 on centre 1
    at a grid radius equals the grid value times sqrt(1/4pi) (basis_norm, numerical branch)."""
    meta, _, gx, gv = fx
    s = S.c2_bfd_example()
    o = oracle_mod.Oracle(s)
    c0 = np.array(meta["cent"][0])
    d = np.array([0.3, -0.5, 0.8]) / np.linalg.norm([0.3, -0.5, 0.8])
    for i in (1, 57, 400, 1200, 1998):
        phi = o.basis(c0 + gx[i] * d)
        assert abs(phi[0, 0] - gv[0, i] / np.sqrt(4 * np.pi)) <= 1e-12 * max(1e-3, abs(gv[0, i]))
    # beyond the grid (20 bohr) the exponential continuation decays smoothly
    far = [o.basis(c0 + r * d)[0, 0] for r in (20.5, 21.0, 22.0)]
    assert 0 < far[2] < far[1] < far[0]


def test_numerical_basis_derivatives_match_finite_differences(oracle_mod):
    s = S.c2_bfd_example()
    o = oracle_mod.Oracle(s)
    rng = np.random.default_rng(4)
    h = 1e-4
    for _ in range(4):
        pt = np.array(s.cent[0]) + rng.normal(0, 0.8, 3)
        phi = o.basis(pt)
        for k in range(3):
            dp = np.zeros(3); dp[k] = h
            fd = (o.basis(pt + dp)[:, 0] - o.basis(pt - dp)[:, 0]) / (2 * h)
            assert np.allclose(phi[:, 1 + k], fd, rtol=1e-5, atol=1e-7)
        hl = 1e-3
        lap = sum((o.basis(pt + e)[:, 0] + o.basis(pt - e)[:, 0] - 2 * phi[:, 0]) / hl ** 2
                  for e in np.eye(3) * hl)
        assert np.allclose(phi[:, 4], lap, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("nq,exact_deg", [(4, 2), (6, 3), (12, 5), (18, 5), (20, 5), (24, 7), (26, 7), (32, 9),
                                          (50, 11), (86, 15)])
def test_quadrature_rules(oracle_mod, nq, exact_deg):
    """gesqua rules: unit vectors, weights summing to one, and exact integration of the
    Legendre polynomials P_L(u.q) for L <= the rule's degree (sum_q w_q P_L = delta_L0)."""
    s = S.c2_bfd_example()
    s.nquad = nq
    o = oracle_mod.Oracle(s)
    q = o.quadrature()
    assert q.shape[0] == nq
    assert np.allclose(np.linalg.norm(q[:, :3], axis=1), 1.0, atol=1e-12)
    assert abs(q[:, 3].sum() - 1.0) < 1e-9
    from numpy.polynomial import legendre
    u = np.array([0.21, -0.47, 0.856])
    u /= np.linalg.norm(u)
    for L in range(1, exact_deg + 1):
        pl = legendre.legval(q[:, :3] @ u, [0] * L + [1])
        assert abs(np.dot(q[:, 3], pl)) < 1e-8, (nq, L)


@pytest.mark.parametrize("run", [1, 10])
def test_transcript_een_coefficients_satisfy_the_cusp_conditions(oracle_mod, fx, run):
    """The printed e-e-n coefficients already obey cuspexact4: re-deriving the dependent ones
    from the free ones changes nothing."""
    meta = fx[0]
    s = S.c2_bfd_example(run)
    o = oracle_mod.Oracle(s)
    c = o.een_coefficients()[0]
    ref = np.array(meta["runs"][run]["params"]["c"])
    assert np.allclose(c, ref, rtol=1e-8, atol=1e-9)


def test_oracle_vmc_matches_the_transcript(oracle_mod, fx):
    """VMC with the oracle, the Jastrow of the transcript's second run (e-n, e-e and e-e-n
    terms all non-zero): E = -10.9806973 +- 0.0062221 Ha after 11100 passes."""
    meta = fx[0]
    ref = meta["runs"][1]
    s = S.c2_bfd_example(1)
    o = oracle_mod.Oracle(s)
    nw, ns = 512, 120
    x = S.initial_walkers(s, nw, seed=3)
    r = o.vmc(x, 30, seed=11, sweep0=0, step=s.step, nthreads=0)
    r = o.vmc(r["x"], ns, seed=11, sweep0=30, step=s.step, nthreads=0)
    ew = r["esum"] / ns
    e, err = ew.mean(), ew.std(ddof=1) / np.sqrt(nw)
    print(f"oracle VMC C2 BFD: E = {e:.5f} +- {err:.5f}, reference {ref['energy']} +- {ref['energy_err']}")
    assert abs(e - ref["energy"]) < 3.5 * np.hypot(err, ref["energy_err"])
