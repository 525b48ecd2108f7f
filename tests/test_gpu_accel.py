"""The accelerated Metropolis mover (champ_set_mover imetro 6; metrop_slat_mov1.f90:82-546, the
reference's default VMC mover) on the GPU against the oracle's restatement of it
(orc_vmc_accel): the same seed and the same counter-based draws give the same walk (FP64; a
walker may split off where an acceptance decision ties at the last bit), and VMC energies of the
reference's examples sampled with it agree with their transcripts.
"""
import json
import os

import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.mark.parametrize("k", [1, 2, "c2bfd"])
def test_accelerated_walk_follows_the_oracle(oracle_mod, k):
    from champ_b200.engine import Engine
    s = S.c2_bfd_example(10) if k == "c2bfd" else S.get_system(k)
    nw = 32
    x = S.initial_walkers(s, nw, seed=18)
    eng = Engine(s, nw, "fp64")
    eng.set_walkers(x)
    eng.set_mover(6, deltar=5.0, deltat=1.0, fbias=1.0)
    st = eng.vmc_sweeps(3, seed=777, sweep0=0, step=0.5)
    xg = eng.get_walkers()
    ref = oracle_mod.Oracle(s).vmc_accel(x, 3, seed=777, sweep0=0, deltar=5.0, deltat=1.0, fbias=1.0, nthreads=4)
    same = np.all(np.abs(xg - ref["x"]) < 1e-9, axis=(1, 2))
    print(f"system {k}: {same.sum()}/{nw} walkers identical; acceptance {st['accept'].sum() / (3 * nw * s.nelec):.3f}")
    assert same.sum() >= nw - 2
    assert np.allclose(st["accept"][same], ref["accept"][same])
    assert np.allclose(st["esum"][same], ref["esum"][same], rtol=1e-8, atol=1e-7)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_accelerated_vmc_be_example_matches_transcript(prec):
    """The reference's Be example with its own mover: E = -14.6463051 +- 0.0075680 Ha."""
    from champ_b200.engine import Engine
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "be_vb1.json")))
    ref = fx["reference"]
    s = S.be_example()
    nw, ns = 4096, 200
    eng = Engine(s, nw, prec)
    eng.set_walkers(S.initial_walkers(s, nw, seed=19))
    eng.set_mover(6)
    eng.vmc_sweeps(60, seed=98, sweep0=0, step=0.5, stats=False)
    st = eng.vmc_sweeps(ns, seed=98, sweep0=60, step=0.5)
    e_w = st["esum"] / ns
    e, err = e_w.mean(), e_w.std(ddof=1) / np.sqrt(nw)
    acc = st["accept"].sum() / (nw * ns * s.nelec)
    print(f"Be example, imetro 6 ({prec}): E = {e:.5f} +- {err:.5f}, acceptance {acc:.3f}; "
          f"reference {ref['energy']} +- {ref['energy_err']}")
    assert abs(e - ref["energy"]) < 3.5 * np.hypot(err, ref["energy_err"]), (e, err)
    # the moves about the nucleus are accepted far more often than Gaussian steps (0.49 here)
    assert acc > 0.7, acc


def test_accelerated_vmc_c2_example_matches_transcript():
    """The reference's final C2 run (its optimised Jastrow) with its own mover: within 3.5
    combined errors of -11.0176327 +- 0.0005000 Ha."""
    from champ_b200.engine import Engine
    meta = S.c2_bfd_fixture()[0]
    ref = meta["runs"][10]
    s = S.c2_bfd_example(10)
    nw, neq, ns = 8192, 60, 200
    eng = Engine(s, nw, "mixed")
    eng.set_walkers(S.initial_walkers(s, nw, seed=210))
    eng.set_mover(6)
    eng.vmc_sweeps(neq, seed=910, sweep0=0, step=s.step, stats=False)
    st = eng.vmc_sweeps(ns, seed=910, sweep0=neq, step=s.step)
    ew = st["esum"] / ns
    e, err = ew.mean(), ew.std(ddof=1) / np.sqrt(nw)
    acc = st["accept"].sum() / (nw * ns * s.nelec)
    z = (e - ref["energy"]) / np.hypot(err, ref["energy_err"])
    print(f"C2 run 10, imetro 6: E = {e:.6f} +- {err:.6f}, acceptance {acc:.3f}; transcript "
          f"{ref['energy']:.7f} +- {ref['energy_err']:.7f}; z = {z:+.2f}")
    assert abs(z) < 3.5


def test_set_mover_validates_and_corrects():
    from champ_b200.engine import Engine, ChampError
    eng = Engine(S.get_system(2), 8, "fp64")
    with pytest.raises(ChampError):
        eng.set_mover(3)
    eng.set_mover(6, deltar=0.5, deltat=3.0, fbias=9.0)  # corrected to 2, 2, 2 as the reference does
    eng.set_walkers(S.initial_walkers(S.get_system(2), 8, seed=1))
    st = eng.vmc_sweeps(2, seed=1, sweep0=0, step=0.5)
    assert np.all(np.isfinite(st["elast"]))


def test_accelerated_mover_drift_from_cached_orbital_rows():
    """Mixed precision, walker state in HBM: the accelerated mover's drift at the current position
    from the last FP64 evaluation's orbital rows (option "mover_cache", kept current by the accepted
    moves) against evaluating the orbitals there again.  The drifts differ at FP32 rounding; the
    accelerated proposal follows the drift and each move changes the next electron's drift, so the
    difference grows through a sweep (first electron: 1e-7 bohr) without changing the sampling:
    after one sweep most walkers agree to 1e-3 bohr and the acceptances agree."""
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=8)
    nw = 128
    x = S.initial_walkers(s, nw, seed=21)
    out = {}
    for cache in (1, 0):
        eng = Engine(s, nw, "mixed")
        eng.set_mover(6)
        eng.set_option("mover_cache", cache)
        assert eng.get_option("mover_cache") == cache
        eng.set_walkers(x)
        st = eng.vmc_sweeps(1, seed=9, sweep0=0, step=s.step)
        out[cache] = (eng.get_walkers(), st)
        eng.close()
    d = np.abs(out[1][0] - out[0][0]).reshape(nw, -1, 3).max(axis=2)
    close = d.max(axis=1) < 1e-3
    acc1, acc0 = out[1][1]["accept"].sum(), out[0][1]["accept"].sum()
    print(f"mover_cache: first electron max {d[:, 0].max():.2e} bohr, {close.mean():.3f} of walkers within "
          f"1e-3 bohr, acceptances {acc1:.0f} / {acc0:.0f}")
    assert np.median(d[:, 0]) < 1e-5
    assert close.mean() >= 0.6
    assert abs(acc1 - acc0) <= 0.02 * acc0
