"""Parameter derivatives on the GPU (C ABI champ_param_grad / champ_accumulate_oh) against
central finite differences (h = 1e-5) of the FP64 oracle's ln|psi| and E_L in each free
parameter -- CSF coefficients, orbital rotations (coefficients of orbital i += h times those of
orbital j) and Jastrow coefficients -- on the same walkers.

Tolerance: |GPU - FD| <= 2e-5 * max(1, |FD|) for d ln psi/dp, and <= 2e-4 * max(1, |E_L|)
for dE_L/dp (FD truncation and cancellation bound the comparison, not the GPU result).
"""
import copy

import numpy as np
import pytest

from champ_b200 import system as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


def cusp_dependents(nordc):
    """Indices fixed by the e-e-n cusp conditions (iwc4 of qmc/fit/cuspinit4.f90)."""
    if nordc <= 1:
        return []
    iwc = [0] * (2 * (nordc - 1))
    i = 0
    for n in range(2, nordc + 1):
        for k in range(n - 1, -1, -1):
            l_hi = n - k - 2 if k == 0 else n - k
            for l in range(l_hi, -1, -1):
                m = (n - k - l) // 2
                if 2 * m != n - k - l:
                    continue
                i += 1
                if k == 1 and iwc[n - 2] == 0:
                    iwc[n - 2] = i
                if k == 0 and iwc[n + nordc - 3] == 0:
                    iwc[n + nordc - 3] = i
    return [v - 1 for v in iwc]


def jastrow_params(s):
    """Free Jastrow parameters in the engine's order: (array name, index)."""
    out = []
    for it in range(s.nctype):
        for k in range(2, s.norda + 1):
            out.append(("a4", (it, k)))
    for isb in range(s.nspin2b):
        for k in range(1, s.nordb + 1):
            out.append(("b", (isb, k)))
    if s.nordc > 1:
        dep = cusp_dependents(s.nordc) if s.een_cusp else []
        nt = S.nterms4(s.nordc)
        for it in range(s.nctype):
            for ll in range(nt):
                if ll not in dep:
                    out.append(("c", (it, ll)))
    return out


def orbital_params(s):
    """Orbital rotations (i, j, antisymmetric) by orbital class, in the order of
    single_ex_wf_bld (qmc/deriv_orb_mod.f90:130-417).  Closed: occupied in both spins of every
    determinant; open/active: occupied somewhere else; virtual: nowhere.  One determinant:
    closed->open, closed->virtual, open->virtual.  Several: closed->active, closed->virtual,
    active i->active j (i < j, antisymmetric), active->virtual."""
    ne, nu = s.nelec, s.nup
    both_all = np.ones(s.norb, bool)
    anyocc = np.zeros(s.norb, bool)
    for det in s.det_orb:
        up, dn = set(int(o) for o in det[:nu]), set(int(o) for o in det[nu:ne])
        for m in range(s.norb):
            both_all[m] &= (m in up) and (m in dn)
            anyocc[m] |= (m in up) or (m in dn)
    cls = [m for m in range(s.norb) if both_all[m]]
    mid = [m for m in range(s.norb) if anyocc[m] and not both_all[m]]
    vir = [m for m in range(s.norb) if not anyocc[m]]
    out = [(i, j, 0) for i in cls for j in mid] + [(i, j, 0) for i in cls for j in vir]
    if s.ndet > 1:
        out += [(mid[a], mid[b], 1) for a in range(len(mid)) for b in range(a + 1, len(mid))]
    out += [(i, j, 0) for i in mid for j in vir]
    return out


def all_params(s):
    """(kind, name, idx) in the engine's order: CSF, orbital rotations, Jastrow."""
    out = []
    if s.ndet > 1:
        out += [("csf", "csf_coef", (q,)) for q in range(1, len(s.csf_coef))]
    out += [("orb", "coef", ij) for ij in orbital_params(s)]
    out += [("jas", name, idx) for name, idx in jastrow_params(s)]
    return out


def perturbed(s, name, idx, h):
    s2 = copy.deepcopy(s)
    arr = getattr(s2, name).copy()
    if name == "coef":  # rotate orbital i towards orbital j (and j away from i)
        i, j, rev = idx
        ai, aj = arr[i].copy(), arr[j].copy()
        arr[i] = ai + h * aj
        if rev:
            arr[j] = aj - h * ai
    else:
        arr[idx] += h
    setattr(s2, name, arr)
    return s2


@pytest.mark.parametrize("k,prec", [(1, "fp64"), (2, "fp64"), (3, "fp64"), (1, "mixed"), (2, "mixed"), (3, "mixed"),
                                    (5, "fp64"), (5, "mixed"), ("c2bfd", "mixed")])
def test_param_derivatives_match_finite_differences(oracle_mod, k, prec):
    """Systems 1-3: every parameter; the 128-electron cluster (2064 parameters) and the
    reference's C2 example (24 Jastrow, 256 orbital-rotation parameters): a seeded subset of 24.
    Mixed precision evaluates the derivatives in FP64 like the FP64 engine."""
    from champ_b200.engine import Engine
    s = S.c2_bfd_example(10) if k == "c2bfd" else S.get_system(k)
    nw = 2 if k in (5, "c2bfd") else 4
    x = S.initial_walkers(s, nw, seed=60 + (9 if k == "c2bfd" else k))
    eng = Engine(s, nw, prec)
    eng.set_walkers(x)
    nj, ncsf, norb = eng.nparam()
    params = all_params(s)
    assert nj == len(jastrow_params(s)) and norb == len(orbital_params(s))
    assert nj + ncsf + norb == len(params)
    dl, de, el = eng.param_grad()
    o0 = oracle_mod.Oracle(s)
    for w in range(nw):
        assert abs(el[w] - o0.eval(x[w])["energy"]) <= 1e-8 * max(1, abs(el[w]))
    h = 1e-5
    sel = range(len(params))
    if k in (5, "c2bfd"):
        rng = np.random.default_rng(17)
        jas0 = len(params) - nj
        sel = sorted(set(rng.choice(jas0, 12, replace=False).tolist()) |
                     set((jas0 + rng.choice(nj, min(12, nj), replace=False)).tolist()))
    for ip in sel:
        kind, name, idx = params[ip]
        op = oracle_mod.Oracle(perturbed(s, name, idx, h))
        om = oracle_mod.Oracle(perturbed(s, name, idx, -h))
        for w in range(nw):
            rp, rm = op.eval(x[w]), om.eval(x[w])
            g_fd = (rp["lnpsi"] - rm["lnpsi"]) / (2 * h)
            e_fd = (rp["energy"] - rm["energy"]) / (2 * h)
            assert abs(dl[w, ip] - g_fd) <= 2e-5 * max(1, abs(g_fd)), (name, idx, w, dl[w, ip], g_fd)
            assert abs(de[w, ip] - e_fd) <= 2e-4 * max(1, abs(el[w])), (name, idx, w, de[w, ip], e_fd)


@pytest.mark.parametrize("k,nw", [(2, 64), (3, 32), (5, 8), ("c2bfd", 64)])
def test_forward_backward_pair_matches_fused_pass(k, nw):
    """champ_param_grad_fwd + champ_param_grad_bwd (the reverse sweep over the tape) against the
    one-pass evaluation (option param_grad_mode 1) on the same walkers: FP64 to 1e-9 relative;
    the mixed engine's FP32 reverse sweep to 1e-5 of max(1, |value|) for d ln psi/dp and 3e-3 of
    max(1, |E_L|) for dE_L/dp (measured: 1e-5 on the dimers, 6e-4 on the cluster, 1.5e-3 on the C2
    example, where the nonlocal part subtracts each parameter's basis function at the electron's
    position from its values at the quadrature points in FP32), with E_L itself identical to the
    FP64 engine's."""
    from champ_b200.engine import Engine
    s = S.c2_bfd_example(10) if k == "c2bfd" else S.get_system(k)
    x = S.initial_walkers(s, nw, seed=90)
    e64 = Engine(s, nw, "fp64")
    e64.set_walkers(x)
    e64.set_option("param_grad_mode", 1)
    dl1, de1, el1 = e64.param_grad()
    e64.set_option("param_grad_mode", 0)
    el0 = e64.param_grad_fwd()
    dl0, de0 = e64.param_grad_bwd()
    assert np.allclose(el0, el1, rtol=1e-12, atol=1e-12)
    sc = np.maximum(1.0, np.abs(el1))[:, None]
    assert np.all(np.abs(dl0 - dl1) <= 1e-9 * np.maximum(1.0, np.abs(dl1)))
    assert np.all(np.abs(de0 - de1) <= 1e-9 * sc)
    with pytest.raises(Exception):
        e64.param_grad_bwd()  # the tape was consumed
    em = Engine(s, nw, "mixed")
    em.set_walkers(x)
    dlm, dem, elm = em.param_grad()
    assert np.all(np.abs(elm - el1) <= 1e-6)
    ed = float(np.max(np.abs(dlm - dl1) / np.maximum(1.0, np.abs(dl1))))
    ee = float(np.max(np.abs(dem - de1) / sc))
    print(f"system {k}: mixed reverse sweep vs FP64: d ln psi/dp {ed:.2e}, dE_L/dp {ee:.2e} (relative)")
    assert ed <= 1e-5 and ee <= 3e-3, (ed, ee)


def test_oh_accumulation_matches_numpy():
    from champ_b200.engine import Engine
    s = S.c2_dimer()
    nw = 256
    eng = Engine(s, nw, "fp64")
    eng.set_walkers(S.initial_walkers(s, nw, seed=3))
    dl, de, el = eng.param_grad()
    wt = np.random.default_rng(1).uniform(0.5, 1.5, nw)
    Sm, Hm = eng.accumulate_oh(wt)
    Oa = np.hstack([np.ones((nw, 1)), dl])
    Mb = np.hstack([el[:, None], el[:, None] * dl + de])
    assert np.allclose(Sm, (Oa * wt[:, None]).T @ Oa, rtol=1e-12, atol=1e-9)
    assert np.allclose(Hm, (Oa * wt[:, None]).T @ Mb, rtol=1e-12, atol=1e-7)


def test_oh_device_buffers_match_host_copy():
    """champ_oh_buffers exposes the same accumulators champ_accumulate_oh copies to the host (the
    device tensors the multi-rank all-reduce sums in place)."""
    import torch
    from champ_b200.engine import Engine
    from champ_b200.dist import oh_tensors, reduce_oh
    s = S.c2_dimer()
    nw = 128
    eng = Engine(s, nw, "fp64")
    eng.set_walkers(S.initial_walkers(s, nw, seed=4))
    eng.param_grad()
    Sh, Hh = eng.accumulate_oh()
    Sd, Hd = oh_tensors(eng)
    torch.cuda.synchronize()
    assert np.array_equal(Sd.cpu().numpy(), Sh) and np.array_equal(Hd.cpu().numpy(), Hh)
    Sr, Hr = reduce_oh(eng)  # one rank: unchanged
    assert np.array_equal(Sr.cpu().numpy(), Sh)


@pytest.mark.parametrize("k", [1, 2, 3, "c2bfd", "be"])
def test_jastrow_derivatives_match_oracle_analytic(oracle_mod, k):
    """The Jastrow block of champ_param_grad (forward pass + reverse sweep, FP64) against the
    oracle's analytic restatement of deriv_jastrow4 and deriv_nonloc_pot
    (orc_jastrow_param_grad, itself pinned to finite differences in
    tests/test_oracle_jastrow_derivs.py): 1e-9 of max(1, |value|) for d ln psi/dp and of
    max(1, |E_L|) for dE_L/dp."""
    from champ_b200.engine import Engine
    if k == "c2bfd":
        s = S.c2_bfd_example(10)
    elif k == "be":
        s = S.be_example()
    else:
        s = S.get_system(k)
    nw = 8
    x = S.initial_walkers(s, nw, seed=77)
    eng = Engine(s, nw, "fp64")
    eng.set_walkers(x)
    nj, ncsf, norb = eng.nparam()
    dl, de, el = eng.param_grad()
    o = oracle_mod.Oracle(s)
    for w in range(nw):
        rl, re_ = o.jastrow_param_grad(x[w])
        assert len(rl) == nj
        gl, ge = dl[w, ncsf + norb:], de[w, ncsf + norb:]
        assert np.all(np.abs(gl - rl) <= 1e-9 * np.maximum(1.0, np.abs(rl))), np.abs(gl - rl).max()
        assert np.all(np.abs(ge - re_) <= 1e-9 * max(1.0, abs(el[w]))), np.abs(ge - re_).max()
