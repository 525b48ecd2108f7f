"""The oracle's analytic Jastrow parameter derivatives (orc_jastrow_param_grad: a restatement of
deriv_jastrow4's gvalue, g and d2g, qmc/vmc/deriv_jastrow4.f90, and of the nonlocal part of
deriv_nonloc_pot, qmc/fit/deriv_nonloc_pot.f90) against central finite differences of the
oracle's own ln|psi| and E_L (h = 1e-5) -- the check that pins the analytic restatement before
the GPU is compared with it (tests/test_gpu_pgrad.py).  CPU only.

Tolerance: FD truncation and cancellation: 1e-6 of max(1, |FD|) for d ln psi/dp, 2e-5 of
max(1, |E_L|) for dE_L/dp.
"""
import copy

import numpy as np
import pytest

from champ_b200 import system as S


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
    out = [("a4", (it, k)) for it in range(s.nctype) for k in range(2, s.norda + 1)]
    out += [("b", (isb, k)) for isb in range(s.nspin2b) for k in range(1, s.nordb + 1)]
    if s.nordc > 1:
        dep = cusp_dependents(s.nordc) if s.een_cusp else []
        out += [("c", (it, ll)) for it in range(s.nctype) for ll in range(S.nterms4(s.nordc)) if ll not in dep]
    return out


def perturbed(s, name, idx, h):
    s2 = copy.deepcopy(s)
    arr = getattr(s2, name).copy()
    arr[idx] += h
    setattr(s2, name, arr)
    return s2


@pytest.mark.parametrize("k", [1, 2, 3, "c2bfd", "be"])
def test_oracle_jastrow_derivatives_match_fd(k):
    from oracle import oracle
    oracle.build()
    if k == "c2bfd":
        s = S.c2_bfd_example(10)
    elif k == "be":
        s = S.be_example()
    else:
        s = S.get_system(k)
    x = S.initial_walkers(s, 2, seed=41)
    o = oracle.Oracle(s)
    params = jastrow_params(s)
    h = 1e-5
    for w in range(2):
        dl, de = o.jastrow_param_grad(x[w])
        assert len(dl) == len(params)
        el = o.eval(x[w])["energy"]
        for ip, (name, idx) in enumerate(params):
            rp = oracle.Oracle(perturbed(s, name, idx, h)).eval(x[w])
            rm = oracle.Oracle(perturbed(s, name, idx, -h)).eval(x[w])
            g_fd = (rp["lnpsi"] - rm["lnpsi"]) / (2 * h)
            e_fd = (rp["energy"] - rm["energy"]) / (2 * h)
            assert abs(dl[ip] - g_fd) <= 1e-6 * max(1, abs(g_fd)), (name, idx, dl[ip], g_fd)
            assert abs(de[ip] - e_fd) <= 2e-5 * max(1, abs(el)), (name, idx, de[ip], e_fd)


def test_pderiv_gradients_match_fd_of_the_jastrow():
    """d grad_i J/dp and d sum lap J/dp: the b_2 (Pade) parameter and a linear one, against FD
    of the oracle's Jastrow gradient and Laplacian."""
    from oracle import oracle
    s = S.get_system(2)
    x = S.initial_walkers(s, 1, seed=5)[0]
    o = oracle.Oracle(s)
    g, gv, d2 = o.jastrow_pderiv(x)
    params = jastrow_params(s)
    h = 1e-5
    for ip, (name, idx) in enumerate(params):
        if not (name == "b" and idx[1] in (1, 2)) and name != "c":
            continue
        vp, vm = np.zeros((s.nelec, 3)), np.zeros((s.nelec, 3))
        op, om = oracle.Oracle(perturbed(s, name, idx, h)), oracle.Oracle(perturbed(s, name, idx, -h))
        jp, vp, lp = op.jastrow(x)
        jm, vm, lm = om.jastrow(x)
        assert abs(g[ip] - (jp - jm) / (2 * h)) <= 1e-6 * max(1, abs(g[ip]))
        assert np.allclose(gv[ip], (vp - vm) / (2 * h), rtol=1e-5, atol=1e-6)
        assert abs(d2[ip] - (lp - lm) / (2 * h)) <= 1e-5 * max(1, abs(d2[ip]))
