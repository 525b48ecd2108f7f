"""ctypes binding of the engine's C ABI (include/champ_b200.h).

``Engine`` mirrors the reference's per-walker interface for all walkers at once:
``eval_full`` ~ hpsi, ``propose_1e`` ~ hpsie, ``accept_1e`` ~ jassav+detsav+dete_save,
``grad_1e`` ~ eval_grad, ``set_walkers`` ~ psi_at, ``vmc_sweeps`` ~ the metrop sweep loop.
Errors raise ``ChampError`` carrying the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .system import System

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchamp_b200.so")

EXPORTED_SYMBOLS = [
    "champ_last_error", "champ_version", "champ_create", "champ_destroy", "champ_nparam",
    "champ_set_walkers", "champ_get_walkers", "champ_set_quadrature_rotation", "champ_eval_full",
    "champ_propose_1e", "champ_accept_1e", "champ_grad_1e", "champ_vmc_sweeps", "champ_vmc_run_host",
    "champ_walker_status", "champ_synchronize", "champ_param_grad", "champ_accumulate_oh",
    "champ_dmc_init", "champ_dmc_steps", "champ_num_walkers", "champ_eval_energy_noalloc", "champ_set_option",
    "champ_get_option", "champ_oh_buffers", "champ_phase_times", "champ_param_grad_fwd", "champ_param_grad_bwd",
    "champ_linear_update", "champ_set_params", "champ_get_params", "champ_apply_param_step",
    "champ_check_param_step", "champ_eval_param_step", "champ_linear_method_step", "champ_autotune",
    "champ_set_mover", "champ_tmoves",
]

PREC = {"fp64": 0, "mixed": 1, "fp32": 2}

_lib = None


class ChampError(RuntimeError):
    pass


class EvalOut(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("lnpsi", "sign", "psij", "velocity", "div_v", "d2lnpsi", "pe", "pe_ee", "pe_nonloc", "energy")]


class VmcStats(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("esum", "e2sum", "accept", "elast")]


def load_library(path: str = LIB_PATH):
    """Load the CUDA engine.  Raises if the library has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ChampError(f"engine library not built: {path} (run python -m champ_b200.build)")
    L = C.CDLL(path)
    vp, i32, dp, u64 = C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_uint64
    L.champ_last_error.restype = C.c_char_p
    L.champ_version.restype = C.c_char_p
    L.champ_create.argtypes = [vp, i32, i32, vp, C.POINTER(vp)]
    L.champ_destroy.argtypes = [vp]
    L.champ_nparam.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
    L.champ_set_walkers.argtypes = [vp, i32, dp]
    L.champ_get_walkers.argtypes = [vp, dp]
    L.champ_set_quadrature_rotation.argtypes = [vp, dp]
    L.champ_eval_full.argtypes = [vp, C.POINTER(EvalOut)]
    L.champ_propose_1e.argtypes = [vp, i32, dp, dp, dp]
    L.champ_accept_1e.argtypes = [vp, i32, C.POINTER(C.c_uint8)]
    L.champ_grad_1e.argtypes = [vp, i32, dp]
    L.champ_vmc_sweeps.argtypes = [vp, i32, u64, u64, C.c_double, C.POINTER(VmcStats)]
    L.champ_vmc_run_host.argtypes = [vp, i32, dp, i32, u64, u64, C.c_double, dp]
    L.champ_walker_status.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.champ_synchronize.argtypes = [vp]
    L.champ_param_grad.argtypes = [vp, dp, dp, dp]
    L.champ_accumulate_oh.argtypes = [vp, dp, dp, dp]
    L.champ_dmc_init.argtypes = [vp, i32, C.c_double, C.c_double]
    L.champ_dmc_steps.argtypes = [vp, i32, u64, dp]
    L.champ_num_walkers.argtypes = [vp, C.POINTER(i32)]
    L.champ_eval_energy_noalloc.argtypes = [vp, i32, vp, vp]
    L.champ_set_option.argtypes = [vp, C.c_char_p, C.c_int64]
    L.champ_get_option.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int64)]
    L.champ_oh_buffers.argtypes = [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    L.champ_phase_times.argtypes = [vp, dp, C.POINTER(i32)]
    L.champ_param_grad_fwd.argtypes = [vp, dp]
    L.champ_param_grad_bwd.argtypes = [vp, dp, dp]
    L.champ_linear_update.argtypes = [i32, i32, dp, dp, C.c_double, C.c_double, i32, dp, dp]
    L.champ_set_params.argtypes = [vp, dp, dp, dp, dp, dp]
    L.champ_get_params.argtypes = [vp, dp, dp, dp, dp, dp]
    L.champ_apply_param_step.argtypes = [vp, dp]
    L.champ_check_param_step.argtypes = [vp, dp, C.c_double, C.POINTER(i32)]
    L.champ_eval_param_step.argtypes = [vp, dp, dp, dp]
    L.champ_linear_method_step.argtypes = [vp, i32, C.POINTER(i32), dp, dp, C.c_double, C.c_double, dp, dp, dp]
    L.champ_autotune.argtypes = [vp, i32, u64, C.c_double, C.c_char_p, C.c_char_p, i32]
    L.champ_set_mover.argtypes = [vp, i32, C.c_double, C.c_double, C.c_double]
    L.champ_tmoves.argtypes = [vp, u64, u64, C.c_double, i32, C.POINTER(i32)]
    for n in EXPORTED_SYMBOLS:
        if n not in ("champ_last_error", "champ_version"):
            getattr(L, n).restype = C.c_int
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def linear_update(S, H, ncsf=0, sigma=0.0, diag_stab=0.0, select=0):
    """champ_linear_update: parameter variations of the linear method from the O/H sums."""
    L = load_library()
    S = np.ascontiguousarray(S, np.float64)
    H = np.ascontiguousarray(H, np.float64)
    P = S.shape[0] - 1
    dp, info = np.zeros(P), np.zeros(4)
    rc = L.champ_linear_update(P, ncsf, _p(S), _p(H), sigma, diag_stab, select, _p(dp), _p(info))
    if rc != 0:
        raise ChampError(f"champ error {rc}: {L.champ_last_error().decode()}")
    return dp, info


class Engine:
    """One engine context (one system, up to w_max walkers, one precision)."""

    def __init__(self, system: System, w_max: int, precision: str = "fp64", stream: int = 0):
        self.lib = load_library()
        self.system = system
        self.N = system.nelec
        self.w_max = w_max
        self._cs, self._keep = system.to_c()
        h = C.c_void_p()
        self._check(self.lib.champ_create(C.byref(self._cs), w_max, PREC[precision], C.c_void_p(stream), C.byref(h)))
        self.h = h
        self.nw = 0

    def _check(self, rc):
        if rc != 0:
            raise ChampError(f"champ error {rc}: {self.lib.champ_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.champ_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- walkers
    def set_walkers(self, x):
        x = np.ascontiguousarray(x, np.float64)
        self.nw = x.shape[0]
        self._check(self.lib.champ_set_walkers(self.h, self.nw, _p(x)))

    def get_walkers(self):
        x = np.zeros((self.nw, self.N, 3))
        self._check(self.lib.champ_get_walkers(self.h, _p(x)))
        return x

    def set_rotation(self, rot=None):
        if rot is None:
            self._check(self.lib.champ_set_quadrature_rotation(self.h, None))
        else:
            r = np.ascontiguousarray(rot, np.float64)
            self._check(self.lib.champ_set_quadrature_rotation(self.h, _p(r)))

    # -- hpsi
    def eval_full(self):
        nw, N = self.nw, self.N
        out = {k: np.zeros(nw) for k in ("lnpsi", "sign", "psij", "d2lnpsi", "pe", "pe_ee", "pe_nonloc", "energy")}
        out["velocity"] = np.zeros((nw, N, 3))
        out["div_v"] = np.zeros((nw, N))
        eo = EvalOut(**{k: _p(v) for k, v in out.items()})
        self._check(self.lib.champ_eval_full(self.h, C.byref(eo)))
        return out

    # -- single-electron moves
    def propose_1e(self, iel, xnew, grad=False):
        xnew = np.ascontiguousarray(xnew, np.float64).reshape(self.nw, 3)
        ratio = np.zeros(self.nw)
        g = np.zeros((self.nw, 3)) if grad else None
        self._check(self.lib.champ_propose_1e(self.h, iel, _p(xnew), _p(ratio), _p(g) if grad else None))
        return (ratio, g) if grad else ratio

    def accept_1e(self, iel, accept):
        a = np.ascontiguousarray(accept, np.uint8)
        self._check(self.lib.champ_accept_1e(self.h, iel, a.ctypes.data_as(C.POINTER(C.c_uint8))))

    def grad_1e(self, iel):
        g = np.zeros((self.nw, 3))
        self._check(self.lib.champ_grad_1e(self.h, iel, _p(g)))
        return g

    # -- VMC
    def vmc_sweeps(self, nsweep, seed, sweep0=0, step=0.5, stats=True):
        if not stats:
            self._check(self.lib.champ_vmc_sweeps(self.h, nsweep, seed, sweep0, step, None))
            return None
        out = {k: np.zeros(self.nw) for k in ("esum", "e2sum", "accept", "elast")}
        st = VmcStats(**{k: _p(v) for k, v in out.items()})
        self._check(self.lib.champ_vmc_sweeps(self.h, nsweep, seed, sweep0, step, C.byref(st)))
        return out

    def vmc_run_host(self, x, nsweep, seed, sweep0=0, step=0.5):
        x = np.ascontiguousarray(x, np.float64).copy()
        nw = x.shape[0]
        el = np.zeros(nw)
        self._check(self.lib.champ_vmc_run_host(self.h, nw, _p(x), nsweep, seed, sweep0, step, _p(el)))
        self.nw = nw
        return x, el

    def nparam(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.lib.champ_nparam(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def param_grad(self, host=True):
        """d ln psi/dp, dE_L/dp (walkers x P) and E_L at the current positions."""
        P = sum(self.nparam())
        if not host:
            self._check(self.lib.champ_param_grad(self.h, None, None, None))
            return None
        dl, de, el = np.zeros((self.nw, P)), np.zeros((self.nw, P)), np.zeros(self.nw)
        self._check(self.lib.champ_param_grad(self.h, _p(dl), _p(de), _p(el)))
        return dl, de, el

    def param_grad_fwd(self, host=True):
        """Forward pass: E_L at the current positions and the tape for param_grad_bwd."""
        el = np.zeros(self.nw) if host else None
        self._check(self.lib.champ_param_grad_fwd(self.h, _p(el) if host else None))
        return el

    def param_grad_bwd(self, host=True):
        """Reverse sweep from the tape: d ln psi/dp and dE_L/dp (walkers x P)."""
        if not host:
            self._check(self.lib.champ_param_grad_bwd(self.h, None, None))
            return None
        P = sum(self.nparam())
        dl, de = np.zeros((self.nw, P)), np.zeros((self.nw, P))
        self._check(self.lib.champ_param_grad_bwd(self.h, _p(dl), _p(de)))
        return dl, de

    def get_params(self):
        """Current parameters: a4, b, c (cusp conditions applied), csf_coef, coef."""
        s = self.system
        from .system import nterms4
        a = np.zeros_like(s.a4, dtype=float)
        b = np.zeros_like(s.b, dtype=float)
        c = np.zeros((s.nctype, nterms4(s.nordc)))
        csf = np.zeros(len(s.csf_coef))
        coef = np.zeros_like(s.coef, dtype=float)
        self._check(self.lib.champ_get_params(self.h, _p(a), _p(b), _p(c) if c.size else None, _p(csf), _p(coef)))
        return dict(a4=a, b=b, c=c, csf_coef=csf, coef=coef)

    def set_params(self, a4=None, b=None, c=None, csf_coef=None, coef=None):
        arr = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (a4, b, c, csf_coef, coef)]
        self._check(self.lib.champ_set_params(self.h, *[None if v is None or v.size == 0 else _p(v) for v in arr]))

    def apply_param_step(self, dp):
        dp = np.ascontiguousarray(dp, np.float64)
        self._check(self.lib.champ_apply_param_step(self.h, _p(dp)))

    def tmoves(self, seed, step, tau, variant=2):
        """champ_tmoves: T-moves of every electron; returns the accepted moves per walker."""
        moved = np.zeros(self.nw, np.int32)
        self._check(self.lib.champ_tmoves(self.h, seed, step, tau, variant, moved.ctypes.data_as(C.POINTER(C.c_int32))))
        return moved

    def set_mover(self, imetro, deltar=5.0, deltat=1.0, fbias=1.0):
        """champ_set_mover: 1 Gaussian steps, 6 the accelerated Metropolis method."""
        self._check(self.lib.champ_set_mover(self.h, imetro, deltar, deltat, fbias))

    def autotune(self, nsweep=2, seed=1, step=None, cache=None):
        """champ_autotune: picks the fastest launch options on the current walkers; returns the
        one-line report."""
        buf = C.create_string_buffer(1024)
        st = self.system.step if step is None else step
        self._check(self.lib.champ_autotune(self.h, nsweep, seed, st, cache.encode() if cache else None, buf, 1024))
        return buf.value.decode()

    def check_param_step(self, dp, psi_lin_var_norm=0.0):
        """champ_check_param_step: 0 (good), 1 (bad) or 2 (bad for any stabilisation)."""
        dp = np.ascontiguousarray(dp, np.float64)
        bad = C.c_int32()
        self._check(self.lib.champ_check_param_step(self.h, _p(dp), psi_lin_var_norm, C.byref(bad)))
        return bad.value

    def eval_param_step(self, dp):
        """Correlated sampling of a trial step: (E_L, ln|psi_new| - ln|psi_old|) of every walker."""
        dp = np.ascontiguousarray(dp, np.float64)
        el, dl = np.zeros(self.nw), np.zeros(self.nw)
        self._check(self.lib.champ_eval_param_step(self.h, _p(dp), _p(el), _p(dl)))
        return el, dl

    def linear_method_step(self, S, H, sigma, diag_stab, sel=None, p_var=0.0):
        """champ_linear_method_step: one stabilised linear-method iteration on the parameters sel
        (S, H: the sums over those parameters).  Returns (dp, final diag_stab, info[8])."""
        S = np.ascontiguousarray(S, np.float64)
        H = np.ascontiguousarray(H, np.float64)
        P = sum(self.nparam())
        dp, info = np.zeros(P), np.zeros(8)
        st = C.c_double(diag_stab)
        if sel is None:
            nsel, psel = P, None
        else:
            sel = np.ascontiguousarray(sel, np.int32)
            nsel, psel = len(sel), sel.ctypes.data_as(C.POINTER(C.c_int32))
        if S.shape != (nsel + 1, nsel + 1) or H.shape != S.shape:
            raise ValueError("S and H must be (nsel+1)^2")
        self._check(self.lib.champ_linear_method_step(self.h, nsel, psel, _p(S), _p(H), sigma, p_var, C.byref(st),
                                                      _p(dp), _p(info)))
        return dp, st.value, info

    def accumulate_oh(self, weights=None):
        P1 = sum(self.nparam()) + 1
        S, H = np.zeros((P1, P1)), np.zeros((P1, P1))
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        self._check(self.lib.champ_accumulate_oh(self.h, _p(w) if w is not None else None, _p(S), _p(H)))
        return S, H

    def oh_buffers(self):
        """Device addresses of the S and H accumulators ((P+1)^2 FP64 each, row-major)."""
        S, H = C.c_void_p(), C.c_void_p()
        self._check(self.lib.champ_oh_buffers(self.h, C.byref(S), C.byref(H)))
        return S.value, H.value

    def dmc_init(self, w_target, tau, gpop=10.0):
        self._check(self.lib.champ_dmc_init(self.h, w_target, tau, gpop))

    def dmc_steps(self, nstep, seed):
        """Runs nstep DMC steps; returns per-step [population, sum w, sum w E_L, E_T]."""
        st = np.zeros((nstep, 4))
        self._check(self.lib.champ_dmc_steps(self.h, nstep, seed, _p(st)))
        nw = C.c_int32()
        self._check(self.lib.champ_num_walkers(self.h, C.byref(nw)))
        self.nw = nw.value
        return st

    def population(self):
        return self.nw

    def walker_status(self):
        f = np.zeros(self.nw, np.uint32)
        self._check(self.lib.champ_walker_status(self.h, f.ctypes.data_as(C.POINTER(C.c_uint32))))
        return f

    def set_option(self, name: str, value: int):
        self._check(self.lib.champ_set_option(self.h, name.encode(), int(value)))

    def get_option(self, name: str) -> int:
        v = C.c_int64()
        self._check(self.lib.champ_get_option(self.h, name.encode(), C.byref(v)))
        return v.value

    def synchronize(self):
        self._check(self.lib.champ_synchronize(self.h))

    def phase_times(self):
        """Device ms and launch counts of the VMC sweep kernels since the last call (option
        "phase_timing" on): {"sweep", "moves", "eval"} -> (ms, launches)."""
        ms = np.zeros(4)
        n = (C.c_int32 * 4)()
        self._check(self.lib.champ_phase_times(self.h, _p(ms), n))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(("sweep", "moves", "eval"))}
