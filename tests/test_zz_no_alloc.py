"""champ_eval_energy_noalloc: local energies for callers that cannot allocate device memory.

Host codes whose GPU memory is owned entirely by their own pool allocator, or that must not
allocate inside a time-critical loop, pass their own device buffers for the walkers and the
energies; the library keeps its intermediates in a fixed device array compiled into it.  This
test calls that entry point through the C ABI with device buffers and compares it, on two calls
in a row with different walkers, with the energies of champ_eval_full on the same walkers,
within the FP64 parity tolerance of the other GPU tests (1e-9 relative to max(1, |E_L|,
|lap ln psi|)).  The file is named to run last in the GPU suite.
"""
import ctypes

import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sysname,nw,prec,tol", [("c2_dimer", 512, "fp64", 1e-9), ("c2_dimer", 512, "mixed", 1e-9),
                                                  ("c2_dimer", 512, "fp32", 1e-6), ("cluster128", 8, "fp64", 1e-9),
                                                  ("cluster128", 8, "mixed", 1e-9), ("cluster128", 8, "fp32", 1e-6)])
def test_noalloc_energy_matches_eval_full_on_two_calls(sysname, nw, prec, tol):
    """c2_dimer keeps each walker's state in shared memory during the evaluation; cluster128
    (128 electrons) keeps it in HBM, here inside the fixed array.  In FP32 precision this entry
    point computes the orbitals on the CUDA cores, so the reference is the same context with the
    tensor-core contraction switched off."""
    import torch
    from champ_b200.engine import Engine
    s = S.c2_dimer() if sysname == "c2_dimer" else S.cluster128()
    eng = Engine(s, nw, prec)
    if prec == "fp32" and sysname == "cluster128":
        eng.set_option("orbital_tc", 0)
    for seed in (11, 12):
        x = S.initial_walkers(s, nw, seed=seed)
        eng.set_walkers(x)
        ref = eng.eval_full()
        xd = torch.from_numpy(x).to("cuda")
        ed = torch.full((nw,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = eng.lib.champ_eval_energy_noalloc(eng.h, nw, ctypes.c_void_p(xd.data_ptr()),
                                               ctypes.c_void_p(ed.data_ptr()))
        assert rc == 0, eng.lib.champ_last_error().decode()
        got = ed.cpu().numpy()
        scale = np.maximum(1.0, np.maximum(np.abs(ref["energy"]), np.abs(ref["d2lnpsi"])))
        assert np.all(np.abs(got - ref["energy"]) <= tol * scale)
        # the context's own walkers are untouched
        assert np.array_equal(eng.get_walkers(), x)


def test_noalloc_rejects_sizes_beyond_the_array():
    import torch
    from champ_b200.engine import Engine
    s = S.c2_dimer()
    eng = Engine(s, 4, "fp64")
    eng.set_walkers(S.initial_walkers(s, 4, seed=1))
    nw = 1 << 22
    xd = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = eng.lib.champ_eval_energy_noalloc(eng.h, nw, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(xd.data_ptr()))
    assert rc == 1 and b"MiB scratch array" in eng.lib.champ_last_error()
