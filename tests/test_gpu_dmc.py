"""Diffusion Monte Carlo on the GPU (champ_dmc_init / champ_dmc_steps).

The Be example wave function of the reference (4 determinants) has a VMC energy of
-14.6463 +- 0.0076 Ha in the reference transcript; its fixed-node DMC energy must lie below
that and above the exact non-relativistic Be energy (-14.66736 Ha) within error bars.  The
population is controlled around its target; FP64 and mixed precision agree statistically.
"""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu

E_EXACT_BE = -14.66736


def run_dmc(system, prec, target, tau, neq, nacc, seed=5, wmax=None):
    from champ_b200.engine import Engine
    eng = Engine(system, wmax or 2 * target, prec)
    eng.set_walkers(S.initial_walkers(system, target, seed=seed))
    eng.vmc_sweeps(50, seed=seed, sweep0=0, step=0.4, stats=False)
    eng.dmc_init(target, tau)
    eng.dmc_steps(neq, seed=seed + 1)
    st = eng.dmc_steps(nacc, seed=seed + 2)
    return eng, st


def block_energy(st, nblock=20):
    e = np.array([b[:, 2].sum() / b[:, 1].sum() for b in np.array_split(st, nblock)])
    return e.mean(), e.std(ddof=1) / np.sqrt(len(e))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dmc_be_example_energy(prec):
    eng, st = run_dmc(S.be_example(), prec, target=4096, tau=0.01, neq=300, nacc=1000)
    e, err = block_energy(st)
    print(f"DMC Be example ({prec}): E = {e:.5f} +- {err:.5f} Ha, population {st[:, 0].min():.0f}..{st[:, 0].max():.0f}")
    pop = st[:, 0]
    assert pop.min() > 0.5 * 4096 and pop.max() < 2 * 4096, (pop.min(), pop.max())
    assert e < -14.6463 - 0.005, (e, err)
    assert e > E_EXACT_BE - 4 * err - 0.002, (e, err)
    assert not eng.walker_status().any()


def test_dmc_c2_population_and_energies_finite():
    eng, st = run_dmc(S.c2_dmc(), "mixed", target=8192, tau=0.01, neq=20, nacc=40, wmax=24576)
    assert np.all(np.isfinite(st))
    assert st[:, 0].min() > 0.3 * 8192 and st[:, 0].max() <= 24576
    assert eng.population() == eng.get_walkers().shape[0]


def test_dmc_graph_replay_matches_step_by_step_launches():
    """The DMC steps replayed as a captured CUDA graph (two steps per replay) follow the same
    trajectory as step-by-step launches: same population per step and the same weights and
    energies (FP64, to summation-order rounding), including an odd step count and a seed change."""
    from champ_b200.engine import Engine
    s = S.c2_dmc()
    out = {}
    for graph in (0, 1):
        eng = Engine(s, 4096, "fp64")
        eng.set_option("dmc_graph", graph)
        assert eng.get_option("dmc_graph") == graph
        eng.set_walkers(S.initial_walkers(s, 2048, seed=9))
        eng.vmc_sweeps(10, seed=9, sweep0=0, step=0.4, stats=False)
        eng.dmc_init(2048, 0.01)
        a = eng.dmc_steps(7, seed=31)
        b = eng.dmc_steps(6, seed=32)
        out[graph] = (np.vstack([a, b]), eng.get_walkers())
    st0, st1 = out[0][0], out[1][0]
    assert np.array_equal(st0[:, 0], st1[:, 0])
    assert np.allclose(st0[:, 1:], st1[:, 1:], rtol=1e-10, atol=1e-10)
    assert np.allclose(out[0][1], out[1][1], rtol=0, atol=1e-12)


def test_dmc_persistent_kernel_matches_warp_per_walker():
    """The persistent DMC step kernel (walkers taken from a work counter) follows the same trajectory
    as the warp-per-walker launch: same populations, weights and energies to summation order."""
    from champ_b200.engine import Engine
    s = S.c2_dmc()
    out = {}
    for persist in (0, 1):
        eng = Engine(s, 4096, "fp64")
        eng.set_option("dmc_persistent", persist)
        assert eng.get_option("dmc_persistent") == persist
        eng.set_walkers(S.initial_walkers(s, 2048, seed=9))
        eng.vmc_sweeps(10, seed=9, sweep0=0, step=0.4, stats=False)
        eng.dmc_init(2048, 0.01)
        out[persist] = (eng.dmc_steps(9, seed=31), eng.get_walkers())
    assert np.array_equal(out[0][0][:, 0], out[1][0][:, 0])
    assert np.allclose(out[0][0][:, 1:], out[1][0][:, 1:], rtol=1e-10, atol=1e-10)
    assert np.allclose(out[0][1], out[1][1], rtol=0, atol=1e-12)


@pytest.mark.parametrize("nvmc", [5, 40])
def test_dmc_population_control_from_short_equilibration(nvmc):
    """Population control from a barely equilibrated start (a few VMC sweeps, near-node outliers
    among the initial local energies): the population stays within a factor of 2 of the target and
    ends within 15 % of it."""
    from champ_b200.engine import Engine
    s = S.c2_dmc()
    target = 8192
    eng = Engine(s, 2 * target, "mixed")
    eng.set_walkers(S.initial_walkers(s, target, seed=11))
    eng.vmc_sweeps(nvmc, seed=5, sweep0=0, step=s.step, stats=False)
    eng.dmc_init(target, 0.01)
    st = eng.dmc_steps(300, seed=3)
    pop = st[:, 0]
    print(f"{nvmc} VMC sweeps: population {pop.min():.0f}..{pop.max():.0f}, last 100 steps {pop[-100:].mean():.0f}")
    assert pop.min() > 0.5 * target and pop.max() < 2 * target
    assert abs(pop[-100:].mean() / target - 1) < 0.15
