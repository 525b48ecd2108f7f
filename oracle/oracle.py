"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, where it is the checker and the timed CPU restatement of the
reference path.  The engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


class OrcEval(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("lnpsi", "sign", "psij", "lnd", "d2lnpsi", "d2j", "d2lnd",
                                          "pe", "pe_ee", "pe_local", "pe_nonloc", "pecent", "energy")] + \
               [(n, C.POINTER(C.c_double)) for n in ("vel", "vj", "vd", "div_v")]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_nterms4.restype = ip
        L.orc_get_c.argtypes = [vp, dp]
        L.orc_set_rotation.argtypes = [vp, dp]
        L.orc_quadrature.argtypes = [vp, dp]
        L.orc_eval_full.restype = ip
        L.orc_eval_full.argtypes = [vp, dp, C.POINTER(OrcEval)]
        L.orc_basis.argtypes = [vp, dp, dp]
        L.orc_orbitals.argtypes = [vp, dp, dp]
        L.orc_jastrow.restype = C.c_double
        L.orc_jastrow.argtypes = [vp, dp, dp, dp]
        L.orc_vps.argtypes = [vp, ip, C.c_double, dp]
        L.orc_ratio_1e.restype = C.c_double
        L.orc_ratio_1e.argtypes = [vp, dp, ip, dp, dp]
        L.orc_philox.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]
        L.orc_random_rotation.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, dp]
        L.orc_jastrow_param_grad.restype = ip
        L.orc_jastrow_param_grad.argtypes = [vp, dp, dp, dp]
        L.orc_jastrow_pderiv.restype = ip
        L.orc_jastrow_pderiv.argtypes = [vp, dp, dp, dp, dp]
        L.orc_tmoves.restype = ip
        L.orc_tmoves.argtypes = [vp, dp, C.c_uint64, C.c_uint32, C.c_uint64, C.c_double, ip]
        L.orc_vmc_accel.restype = ip
        L.orc_vmc_accel.argtypes = [vp, ip, dp, ip, C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                    dp, dp, dp, dp, ip]
        L.orc_vmc.restype = ip
        L.orc_vmc.argtypes = [vp, ip, dp, ip, C.c_uint64, C.c_uint64, C.c_double, dp, dp, dp, dp, ip]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One oracle instance for one system (see champ_b200.system.System)."""

    def __init__(self, system):
        self.system = system
        self._cs, self._keep = system.to_c()
        self.h = lib().orc_create(C.byref(self._cs))
        self.N = system.nelec

    def __del__(self):
        try:
            if self.h:
                lib().orc_destroy(self.h)
        except Exception:
            pass

    def set_rotation(self, rot=None):
        if rot is None:
            lib().orc_set_rotation(self.h, None)
        else:
            r = np.ascontiguousarray(rot, float)
            lib().orc_set_rotation(self.h, _p(r))

    def quadrature(self):
        q = np.zeros((self.system.nquad, 4))
        lib().orc_quadrature(self.h, _p(q))
        return q

    def een_coefficients(self):
        from champ_b200.system import nterms4
        nt = nterms4(self.system.nordc)
        c = np.zeros((self.system.nctype, max(nt, 1)))
        lib().orc_get_c(self.h, _p(c))
        return c[:, :nt]

    def eval(self, x):
        x = np.ascontiguousarray(x, float).reshape(self.N, 3)
        vel = np.zeros((self.N, 3)); vj = np.zeros((self.N, 3)); vd = np.zeros((self.N, 3)); dv = np.zeros(self.N)
        e = OrcEval(vel=_p(vel), vj=_p(vj), vd=_p(vd), div_v=_p(dv))
        sing = lib().orc_eval_full(self.h, _p(x), C.byref(e))
        out = {n: getattr(e, n) for n, _ in OrcEval._fields_[:13]}
        out.update(vel=vel, vj=vj, vd=vd, div_v=dv, singular=bool(sing))
        return out

    def jastrow_param_grad(self, x):
        """Analytic d ln psi/dp and d E_L/dp of the free Jastrow parameters (engine order)."""
        x = np.ascontiguousarray(x, float).reshape(self.N, 3)
        dl, de = np.zeros(4096), np.zeros(4096)
        n = lib().orc_jastrow_param_grad(self.h, _p(x), _p(dl), _p(de))
        if n < 0:
            raise ValueError("singular configuration")
        return dl[:n].copy(), de[:n].copy()

    def jastrow_pderiv(self, x):
        """dJ/dp, d grad_i J/dp [np][N][3] and d sum_i lap_i J/dp of the free Jastrow parameters."""
        x = np.ascontiguousarray(x, float).reshape(self.N, 3)
        g, v, d2 = np.zeros(4096), np.zeros(4096 * 3 * self.N), np.zeros(4096)
        n = lib().orc_jastrow_pderiv(self.h, _p(x), _p(g), _p(v), _p(d2))
        return g[:n].copy(), v[:n * 3 * self.N].reshape(n, self.N, 3).copy(), d2[:n].copy()

    def basis(self, pt):
        pt = np.ascontiguousarray(pt, float)
        phi = np.zeros((self.system.nbasis, 5))
        lib().orc_basis(self.h, _p(pt), _p(phi))
        return phi

    def orbitals(self, pt):
        pt = np.ascontiguousarray(pt, float)
        o = np.zeros((self.system.norb, 5))
        lib().orc_orbitals(self.h, _p(pt), _p(o))
        return o

    def jastrow(self, x):
        x = np.ascontiguousarray(x, float).reshape(self.N, 3)
        v = np.zeros((self.N, 3)); d2 = np.zeros(1)
        val = lib().orc_jastrow(self.h, _p(x), _p(v), _p(d2))
        return val, v, d2[0]

    def vps(self, ict, r):
        v = np.zeros(5)
        lib().orc_vps(self.h, ict, r, _p(v))
        return v[: int(self.system.npotd[ict])]

    def ratio_1e(self, x, iel, xnew):
        x = np.ascontiguousarray(x, float).reshape(self.N, 3)
        xn = np.ascontiguousarray(xnew, float)
        g = np.zeros(3)
        r = lib().orc_ratio_1e(self.h, _p(x), iel, _p(xn), _p(g))
        return r, g

    def vmc(self, x, nsweep, seed, sweep0=0, step=0.5, nthreads=0):
        x = np.ascontiguousarray(x, float).copy()
        nw = x.shape[0]
        es, e2, acc, el = (np.zeros(nw) for _ in range(4))
        lib().orc_vmc(self.h, nw, _p(x), nsweep, seed, sweep0, step, _p(es), _p(e2), _p(acc), _p(el), nthreads)
        return dict(x=x, esum=es, e2sum=e2, accept=acc, elast=el)

    def tmoves(self, x, seed, iw, step, tau, variant=2):
        """T-moves of every electron of one walker; returns (new positions, accepted moves)."""
        x = np.ascontiguousarray(x, float).reshape(self.N, 3).copy()
        n = lib().orc_tmoves(self.h, _p(x), seed, iw, step, tau, variant)
        return x, n

    def vmc_accel(self, x, nsweep, seed, sweep0=0, deltar=5.0, deltat=1.0, fbias=1.0, nthreads=0):
        """VMC with the accelerated Metropolis mover (imetro = 6)."""
        x = np.ascontiguousarray(x, float).copy()
        nw = x.shape[0]
        es, e2, acc, el = (np.zeros(nw) for _ in range(4))
        lib().orc_vmc_accel(self.h, nw, _p(x), nsweep, seed, sweep0, deltar, deltat, fbias, _p(es), _p(e2), _p(acc),
                            _p(el), nthreads)
        return dict(x=x, esum=es, e2sum=e2, accept=acc, elast=el)


def philox(seed, c0, c1, c2, c3):
    o = (C.c_uint32 * 4)()
    lib().orc_philox(seed, c0, c1, c2, c3, o)
    return list(o)


def random_rotation(seed, walker, sweep):
    r = np.zeros(9)
    lib().orc_random_rotation(seed, walker, sweep, _p(r))
    return r.reshape(3, 3)
