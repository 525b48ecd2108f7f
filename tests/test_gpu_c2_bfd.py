"""The reference's C2 pseudopotential example on the GPU engine, through the C ABI.

Per configuration: the FP64 engine against the FP64 oracle (numerical radial basis, BFD
pseudopotential, 6-point quadrature, e-e-n Jastrow of order 5) to 1e-9 relative, and the mixed
engine to the 1e-6 Ha contract.  Statistically: VMC energies against the transcript
(examples/c2_bfd_vtz_rhf_vmc_new.out), whose longest runs carry errors of 5e-4 Ha, each with the
Jastrow parameters that run used (fixture tests/golden/c2_bfd.npz).
"""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.mark.parametrize("run,prec", [(0, "fp64"), (10, "fp64"), (10, "mixed")])
def test_eval_full_matches_oracle(oracle_mod, run, prec):
    from champ_b200.engine import Engine
    s = S.c2_bfd_example(run)
    o = oracle_mod.Oracle(s)
    nw = 48
    x = S.initial_walkers(s, nw, seed=40 + run)
    rot = oracle_mod.random_rotation(5, 2, 9)
    eng = Engine(s, nw, prec)
    eng.set_walkers(x)
    eng.set_rotation(rot)
    g = eng.eval_full()
    o.set_rotation(rot)
    for w in range(nw):
        r = o.eval(x[w])
        sc = max(1.0, abs(r["energy"]), abs(r["d2lnpsi"]))
        assert abs(g["lnpsi"][w] - r["lnpsi"]) <= 1e-9 * max(1, abs(r["lnpsi"])), w
        assert np.allclose(g["velocity"][w], r["vel"], rtol=1e-9, atol=1e-9 * sc)
        assert abs(g["pe_nonloc"][w] - r["pe_nonloc"]) <= 1e-9 * max(1, abs(r["pe_nonloc"]))
        assert abs(g["energy"][w] - r["energy"]) <= min(1e-6, 1e-8 * sc), (w, g["energy"][w], r["energy"])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_vmc_matches_the_transcript(prec):
    """Every transcript run with an error of at most 8e-4 Ha (runs 4-10: the optimisation's later
    iterations and the final VMC run), each with its own Jastrow: |E - E_ref| within 3.5 combined
    standard errors.  8192 walkers x 300 sweeps per run after 80 sweeps of equilibration."""
    from champ_b200.engine import Engine
    meta = S.c2_bfd_fixture()[0]
    nw, neq, ns = 8192, 80, 300
    bad = []
    for run, ref in enumerate(meta["runs"]):
        if ref["energy_err"] > 8e-4:
            continue
        s = S.c2_bfd_example(run)
        eng = Engine(s, nw, prec)
        eng.set_walkers(S.initial_walkers(s, nw, seed=200 + run))
        eng.vmc_sweeps(neq, seed=900 + run, sweep0=0, step=s.step, stats=False)
        st = eng.vmc_sweeps(ns, seed=900 + run, sweep0=neq, step=s.step)
        ew = st["esum"] / ns
        e, err = ew.mean(), ew.std(ddof=1) / np.sqrt(nw)
        sigma = np.sqrt(st["e2sum"].sum() / (nw * ns) - (st["esum"].sum() / (nw * ns)) ** 2)
        z = (e - ref["energy"]) / np.hypot(err, ref["energy_err"])
        print(f"run {run} ({prec}): E = {e:.6f} +- {err:.6f}, sigma {sigma:.4f}; transcript "
              f"{ref['energy']:.7f} +- {ref['energy_err']:.7f}, sigma {ref['sigma']:.5f}; z = {z:+.2f}")
        if abs(z) > 3.5 or abs(sigma - ref["sigma"]) > 0.05:
            bad.append((run, e, err, sigma, z))
        eng.close()
    assert not bad, bad
