"""Delayed inverse updates of the single-electron moves (option "delay_rank": the accepted moves'
rank-1 terms kept aside and folded into the inverse as one FP64 tensor-core product every K
accepted moves of a spin) against updates applied at once, on the 128-electron cluster (walker
state in HBM); and the launch-option autotuner.

Checks: (1) the kept-current inverse -- after equilibrated FP64 sweeps that do not re-invert
(single-kernel evaluation, "reinvert_every" 1000) the sweep's E_L, computed with that inverse,
differs from the oracle's fresh evaluation at the final positions by no more than the same sweeps
with the updates applied at once do (plus 1e-9 relative); (2) the walk -- with and without delay
the same seed moves the walkers alike (the ratios agree to rounding, so at most a rare acceptance
decision near the threshold differs).
"""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


def sweep_errors(rank, nsw=3):
    from champ_b200.engine import Engine
    from oracle import oracle
    s = S.get_system(5)
    nw = 4
    eng = Engine(s, nw, "fp64")
    eng.set_walkers(S.initial_walkers(s, nw, seed=12))
    eng.vmc_sweeps(10, seed=3, sweep0=100, step=s.step, stats=False)  # equilibration (re-inverting)
    eng.set_option("staged_eval", 0)
    eng.set_option("reinvert_every", 1000)
    eng.set_option("delay_rank", rank)
    assert eng.get_option("delay_rank") == rank
    st = eng.vmc_sweeps(nsw, seed=9, sweep0=1, step=s.step)  # sweeps 1..nsw: no re-inversion
    assert st["accept"].min() > 0
    x = eng.get_walkers()
    orc = oracle.Oracle(s)
    return np.array([abs(st["elast"][w] - orc.eval(x[w])["energy"]) / max(1.0, abs(st["elast"][w]))
                     for w in range(nw)])


@pytest.mark.parametrize("rank", [4, 8, 32])
def test_delayed_inverse_as_accurate_as_immediate(rank):
    e0 = sweep_errors(0)
    ek = sweep_errors(rank)
    print(f"rank {rank}: max relative E_L error {ek.max():.2e} (immediate updates {e0.max():.2e})")
    assert ek.max() <= 4 * e0.max() + 1e-9


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_delayed_walk_matches_immediate(prec):
    from champ_b200.engine import Engine
    s = S.get_system(5)
    nw = 64
    x = S.initial_walkers(s, nw, seed=13)
    a, b = Engine(s, nw, prec), Engine(s, nw, prec)
    a.set_walkers(x)
    b.set_walkers(x)
    b.set_option("delay_rank", 0)
    sa = a.vmc_sweeps(2, seed=17, sweep0=0, step=s.step)
    sb = b.vmc_sweeps(2, seed=17, sweep0=0, step=s.step)
    xa, xb = a.get_walkers(), b.get_walkers()
    same = np.all(np.abs(xa - xb) <= 1e-12, axis=(1, 2))
    assert same.mean() >= 0.95, same.mean()
    assert np.allclose(sa["elast"][same], sb["elast"][same], rtol=1e-10, atol=1e-10)
    assert np.array_equal(sa["accept"][same], sb["accept"][same])


def test_delay_rank_option_bounds():
    from champ_b200.engine import Engine, ChampError
    eng = Engine(S.get_system(2), 8, "mixed")  # walker state in shared memory: no delayed updates
    assert eng.get_option("delay_rank") == 0
    with pytest.raises(ChampError):
        eng.set_option("delay_rank", 8)
    e5 = Engine(S.get_system(5), 8, "mixed")
    assert e5.get_option("delay_rank") == 4
    with pytest.raises(ChampError):
        e5.set_option("delay_rank", 33)


def test_autotune_picks_and_caches(tmp_path):
    from champ_b200.engine import Engine
    s = S.get_system(5)
    eng = Engine(s, 64, "mixed")
    eng.set_walkers(S.initial_walkers(s, 64, seed=3))
    cache = str(tmp_path / "tune.txt")
    rep = eng.autotune(nsweep=1, cache=cache)
    assert "delay_rank=" in rep and "staged_eval=" in rep and "move_coop=" in rep, rep
    chosen = dict(kv.split("=") for kv in rep.split(" (")[0].split())
    assert int(chosen["delay_rank"]) == eng.get_option("delay_rank")
    assert int(chosen["staged_eval"]) == eng.get_option("staged_eval")
    assert int(chosen["move_coop"]) == eng.get_option("move_coop")
    # a second context of the same shape takes the choice from the cache, without timing
    e2 = Engine(s, 64, "mixed")
    e2.set_walkers(S.initial_walkers(s, 64, seed=4))
    e2.set_option("delay_rank", 0 if int(chosen["delay_rank"]) else 4)
    rep2 = e2.autotune(nsweep=1, cache=cache)
    assert rep2.startswith("cached:"), rep2
    assert e2.get_option("delay_rank") == int(chosen["delay_rank"])
