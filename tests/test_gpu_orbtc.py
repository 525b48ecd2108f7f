"""Tensor-core orbital contraction (tcgen05, 3-term TF32 split) against the CUDA-core paths.

The full evaluation of an FP32-precision engine whose walker state lives in HBM computes the
orbitals of all electrons of all walkers as one tensor-core product per spin, either fused with
the basis evaluation in shared memory (orbital_tc 1) or from basis rows in HBM (orbital_tc 2).
These tests switch the modes through champ_set_option("orbital_tc") and compare with the
CUDA-core contraction of the same engine (0) and with the FP64 engine: the tensor-core E_L error
relative to max(1, |E_L|, |lap ln psi|) must stay within 3x that of the CUDA-core FP32
contraction (or 1e-6).
"""
import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _scale(ref):
    return np.maximum(1.0, np.maximum(np.abs(ref["energy"]), np.abs(ref["d2lnpsi"])))


def _engines(s, nw, seed):
    from champ_b200.engine import Engine
    x = S.initial_walkers(s, nw, seed=seed)
    e64 = Engine(s, nw, "fp64")
    e64.set_walkers(x)
    em = Engine(s, nw, "fp32")
    return x, e64, em


@pytest.mark.parametrize("ncent", [8, 32])
def test_eval_full_tensor_core_orbitals(ncent):
    s = S.cluster128(ncent=ncent)
    nw = 64 if ncent == 32 else 256
    x, e64, em = _engines(s, nw, 21)
    ref = e64.eval_full()
    out = {}
    for tc in (0, 1, 2):
        em.set_option("orbital_tc", tc)
        assert em.get_option("orbital_tc") == tc
        em.set_walkers(x)
        out[tc] = em.eval_full()
    sc = _scale(ref)
    err = {}
    for tc in (0, 1, 2):
        err[tc] = float(np.max(np.abs(out[tc]["energy"] - ref["energy"]) / sc))
        assert err[tc] <= 2e-3  # the FP32 parity tolerance of the other tests
        lerr = np.abs(out[tc]["lnpsi"] - ref["lnpsi"]) / np.maximum(1.0, np.abs(ref["lnpsi"]))
        assert np.all(lerr <= 1e-5), (tc, float(lerr.max()))
    print(f"cluster ncent={ncent}: max |dE_L|/scale vs FP64: CUDA-core {err[0]:.2e}, "
          f"tensor-core fused {err[1]:.2e}, from basis rows {err[2]:.2e}")
    # the tensor-core contractions are as accurate as the CUDA-core FP32 one
    assert err[1] <= max(3 * err[0], TOL), err
    assert err[2] <= max(3 * err[0], TOL), err
    # no systematic shrinkage of the orbitals: the walker mean of ln|psi| of the chunked
    # tensor-core contractions stays at that of the CUDA-core contraction of the same basis values
    # (accumulated over the whole 464-function K in one TMEM accumulator, the tensor core's
    # truncation moves it by ~1.4e-4 on 32 centres)
    shift = {tc: float(np.mean(out[tc]["lnpsi"] - out[0]["lnpsi"])) for tc in (1, 2)}
    print(f"cluster ncent={ncent}: mean ln psi, tensor-core minus CUDA-core: {shift}")
    assert abs(shift[1]) <= 5e-5 and abs(shift[2]) <= 5e-5, shift


def test_fused_contraction_with_more_tiles_than_sms():
    """1024 walkers x 64 electrons of a spin = 512 tiles of 128 rows per spin, more than the
    148 CTAs of the grid: each CTA carries its stage and barrier-parity counters across several
    tiles.  Both tensor-core paths against the CUDA-core contraction of the same engine."""
    s = S.cluster128(ncent=8)
    nw = 1024
    x, e64, em = _engines(s, nw, 29)
    ref = e64.eval_full()
    sc = _scale(ref)
    out = {}
    for tc in (0, 1, 2):
        em.set_option("orbital_tc", tc)
        em.set_walkers(x)
        out[tc] = em.eval_full()
    e0 = float(np.max(np.abs(out[0]["energy"] - ref["energy"]) / sc))
    for tc in (1, 2):
        err = float(np.max(np.abs(out[tc]["energy"] - ref["energy"]) / sc))
        assert err <= max(3 * e0, TOL), (tc, err, e0)
        shift = float(np.mean(out[tc]["lnpsi"] - out[0]["lnpsi"]))
        assert abs(shift) <= 5e-5, (tc, shift)
        assert np.all(np.isfinite(out[tc]["energy"]))


def test_fused_accumulation_chunks_remove_the_truncation_bias():
    """orbital_tc_chunk 0 (one accumulator over all of K) against the default chunking and
    chunks of one K-block: the walker-mean ln|psi| offset from the CUDA-core contraction of the
    same FP32 basis values (the truncation bias) shrinks with the chunk."""
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=32)
    nw = 256
    x = S.initial_walkers(s, nw, seed=23)
    em = Engine(s, nw, "fp32")
    em.set_option("orbital_tc", 0)
    em.set_walkers(x)
    base = em.eval_full()["lnpsi"]
    em.set_option("orbital_tc", 1)
    assert em.get_option("orbital_tc_chunk") == 4
    shift = {}
    for ch in (0, 4, 1):
        em.set_option("orbital_tc_chunk", ch)
        em.set_walkers(x)
        shift[ch] = abs(float(np.mean(em.eval_full()["lnpsi"] - base)))
    print("mean |ln psi offset from the CUDA-core contraction| by chunk:", shift)
    assert shift[4] < 0.5 * shift[0] and shift[1] < 0.5 * shift[0], shift


def test_vmc_split_sweep_matches_fused_sweep():
    """A VMC sweep run as moves / tensor-core orbitals / E_L gives the walkers of the fused sweep
    (moves do not depend on the E_L) and the same local energies at FP32 tolerance."""
    from champ_b200.engine import Engine
    s = S.cluster128(ncent=8)
    nw = 256
    x = S.initial_walkers(s, nw, seed=5)
    res = {}
    for tc in (0, 1, 2):
        e = Engine(s, nw, "fp32")
        e.set_option("orbital_tc", tc)
        e.set_walkers(x)
        st = e.vmc_sweeps(1, 99, 0, 0.3)
        res[tc] = (e.get_walkers(), st, _scale(e.eval_full()))
    # the starting inverses differ at FP32 rounding level, so a Metropolis decision within that
    # distance of its threshold may differ: compare the walkers whose trajectories coincide
    for tc in (1, 2):
        same = np.all(res[0][0] == res[tc][0], axis=(1, 2))
        assert same.mean() >= 0.98
        assert np.array_equal(res[0][1]["accept"][same], res[tc][1]["accept"][same])
        el0, el1 = res[0][1]["elast"][same], res[tc][1]["elast"][same]
        sc = res[0][2][same]
        assert np.all(np.abs(el0 - el1) <= 1e-5 * sc), (tc, float(np.max(np.abs(el0 - el1) / sc)))


def test_orbital_tc_option_rejected_where_unsupported():
    from champ_b200.engine import Engine, ChampError
    s = S.c2_dimer()
    e = Engine(s, 8, "fp32")
    with pytest.raises(ChampError):
        e.set_option("orbital_tc", 1)
    e.set_option("orbital_tc", 0)
    with pytest.raises(ChampError):
        e.set_option("no_such_option", 1)
