"""FP32 Gaussian moves whose block shares the proposals' coefficient stream (option "move_coop",
block_orbitals) against the same moves with each warp streaming the coefficients itself: the sums
run in the same order, so the walks are identical -- positions, acceptances and energies -- also
when the walker count leaves warps of the last block without a walker."""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nw", [256, 254])
def test_cooperative_moves_walk_the_same_chain(nw):
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=8)
    x = S.initial_walkers(s, nw, seed=17)
    out = {}
    for coop in (1, 0):
        eng = Engine(s, nw, "mixed")
        assert eng.get_option("move_coop") == 1  # on by default for this shape
        eng.set_option("move_coop", coop)
        assert eng.get_option("move_coop") == coop
        eng.set_walkers(x)
        st = eng.vmc_sweeps(3, seed=23, sweep0=0, step=s.step)
        out[coop] = (eng.get_walkers(), st)
        eng.close()
    assert np.array_equal(out[0][0], out[1][0])
    for k in ("accept", "esum", "elast"):
        assert np.array_equal(out[0][1][k], out[1][1][k]), k
    assert out[1][1]["accept"].mean() > 0.1


def test_cooperative_moves_option_bounds():
    from champ_b200.engine import Engine, ChampError
    s = S.get_system(2)  # walker state resident in shared memory: no cooperative moves
    eng = Engine(s, 64, "mixed")
    assert eng.get_option("move_coop") == 0
    with pytest.raises(ChampError):
        eng.set_option("move_coop", 1)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cooperative_orbital_stage_gives_the_same_evaluation(prec):
    """The staged evaluation's orbital part with the block sharing the coefficient stream (option
    "orb_coop") gives the same orbitals, hence bit-identical local energies, as every warp
    streaming the coefficients itself."""
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=8)
    x = S.initial_walkers(s, 96, seed=5)
    out = {}
    for coop in (1, 0):
        eng = Engine(s, 96, prec)
        assert eng.get_option("orb_coop") == 1
        eng.set_option("orb_coop", coop)
        eng.set_walkers(x)
        out[coop] = eng.eval_full()
        eng.close()
    for k in ("energy", "lnpsi", "d2lnpsi", "pe_nonloc", "velocity"):
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("k,prec", [(5, "mixed"), (5, "fp64"), (2, "mixed")])
def test_vmc_run_host_matches_device_sweeps(k, prec):
    """champ_vmc_run_host (walkers from host memory, the state rebuilt without an E_L -- only the
    inverse, log-determinant and move tables for the staged evaluation -- one call of sweeps,
    E_L and walkers back) walks the same chain as set_walkers + champ_vmc_sweeps."""
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=8) if k == 5 else S.get_system(k)
    nw = 64
    x = S.initial_walkers(s, nw, seed=8)
    a = Engine(s, nw, prec)
    a.set_walkers(x)
    st = a.vmc_sweeps(2, seed=13, sweep0=4, step=s.step)
    xa = a.get_walkers()
    b = Engine(s, nw, prec)
    xb, eb = b.vmc_run_host(x, 2, seed=13, sweep0=4, step=s.step)
    assert np.array_equal(xa, xb)
    assert np.array_equal(st["elast"], eb)
