"""The staged full evaluation (four kernels: Jastrow and distances, orbitals per electron, Slater
inversion in shared memory, velocities + pseudopotential + E_L) against the single-kernel
evaluation (option "staged_eval" 0) on the same walkers, and against the FP64 oracle, on systems
whose walker state lives in HBM (the 128-electron cluster, the 36-orbital multi-determinant
dimer).

Tolerance: the two evaluations run the same device code and differ only in the order of
floating-point sums (the inverse, the pair sums): the FP64 parity tolerance, 1e-9 relative, on
E_L, ln|psi| and velocities, among themselves and against the oracle.
"""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu

KEYS = ("energy", "lnpsi", "d2lnpsi", "pe", "pe_nonloc", "psij")


def close(a, b, rtol):
    return np.abs(a - b) <= rtol * np.maximum(1.0, np.abs(b))


def engines(k, nw, prec, seed=3):
    from champ_b200.engine import Engine
    s = S.get_system(k)
    x = S.initial_walkers(s, nw, seed=seed)
    a = Engine(s, nw, prec)
    b = Engine(s, nw, prec)
    if not a.get_option("staged_eval"):
        pytest.skip("walker state of this system is resident in shared memory")
    b.set_option("staged_eval", 0)
    a.set_walkers(x)
    b.set_walkers(x)
    return s, a, b


@pytest.mark.parametrize("k,nw", [(5, 24), (3, 64)])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_staged_matches_single_kernel(k, nw, prec):
    s, a, b = engines(k, nw, prec)
    ea, eb = a.eval_full(), b.eval_full()
    for key in KEYS:
        assert np.all(close(ea[key], eb[key], 1e-9)), (key, np.abs(ea[key] - eb[key]).max())
    assert np.all(close(ea["velocity"], eb["velocity"], 1e-9))
    assert np.all(close(ea["div_v"], eb["div_v"], 1e-9))
    assert np.array_equal(ea["sign"], eb["sign"])
    # after a sweep of moves: the E_L of the staged sweep equals a fresh single-kernel evaluation
    st = a.vmc_sweeps(1, seed=11, sweep0=0, step=s.step)
    x = a.get_walkers()
    b.set_walkers(x)
    b.set_option("reinvert_every", 1)
    eb = b.eval_full()
    ea = a.eval_full()
    assert np.all(close(ea["energy"], eb["energy"], 1e-9))
    assert np.all(np.isfinite(st["elast"]))
    assert a.get_option("launches_per_sweep") == 5


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_staged_cluster_matches_oracle(prec):
    from oracle import oracle
    s, a, _ = engines(5, 4, prec, seed=9)
    a.vmc_sweeps(2, seed=5, sweep0=0, step=0.3, stats=False)
    x = a.get_walkers()
    ea = a.eval_full()
    orc = oracle.Oracle(s)
    for w in range(4):
        r = orc.eval(x[w])
        assert abs(ea["energy"][w] - r["energy"]) <= 1e-9 * max(1.0, abs(r["energy"])), w
        assert abs(ea["lnpsi"][w] - r["lnpsi"]) <= 1e-9 * max(1.0, abs(r["lnpsi"])), w
        assert np.allclose(ea["velocity"][w], r["vel"], rtol=1e-9, atol=1e-9)


def test_staged_vmc_statistics_fp64_vs_single_kernel():
    """The FP64 sweep as moves + staged E_L walks the same chain as the fused sweep kernel
    (identical moves; re-inversion every sweep in both)."""
    s, a, b = engines(5, 64, "fp64", seed=4)
    b.set_option("reinvert_every", 1)
    sa = a.vmc_sweeps(2, seed=21, sweep0=0, step=s.step)
    sb = b.vmc_sweeps(2, seed=21, sweep0=0, step=s.step)
    same = close(sa["esum"], sb["esum"], 1e-8)
    assert same.mean() >= 0.95, same.mean()
    assert np.array_equal(sa["accept"][same], sb["accept"][same])
