"""System descriptors for the engine: the data CHAMP reads from its nuclei, basis,
orbitals, csfs, jastrow and pseudo input blocks, held as numpy arrays and packed
into the C struct ``champ_system`` of include/champ_b200.h.

The five benchmark systems are generated from seeds (``np.random.default_rng(1000+k)``
for system k, with independent sub-streams per ingredient).  They follow the shapes
and value distributions of the benchmark definitions; nothing here is read from a
data set.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

MAX_LCHAN = 5


class ChampSystem(C.Structure):
    """Mirror of ``champ_system`` (include/champ_b200.h)."""

    _fields_ = [
        ("nelec", C.c_int32), ("nup", C.c_int32), ("ncent", C.c_int32), ("nctype", C.c_int32),
        ("cent", C.POINTER(C.c_double)), ("iwctype", C.POINTER(C.c_int32)), ("znuc", C.POINTER(C.c_double)),
        ("nshell", C.c_int32),
        ("shell_cent", C.POINTER(C.c_int32)), ("shell_n", C.POINTER(C.c_int32)),
        ("shell_l", C.POINTER(C.c_int32)), ("shell_kind", C.POINTER(C.c_int32)),
        ("shell_nprim", C.POINTER(C.c_int32)),
        ("prim_zeta", C.POINTER(C.c_double)), ("prim_coef", C.POINTER(C.c_double)),
        ("nbasis", C.c_int32),
        ("basis_shell", C.POINTER(C.c_int32)), ("basis_m", C.POINTER(C.c_int32)),
        ("norb", C.c_int32), ("coef", C.POINTER(C.c_double)),
        ("ndet", C.c_int32), ("det_orb", C.POINTER(C.c_int32)),
        ("ncsf", C.c_int32), ("csf_coef", C.POINTER(C.c_double)), ("csf_ndet", C.POINTER(C.c_int32)),
        ("csf_det", C.POINTER(C.c_int32)), ("csf_det_coef", C.POINTER(C.c_double)),
        ("scalek", C.c_double),
        ("norda", C.c_int32), ("nordb", C.c_int32), ("nordc", C.c_int32), ("nspin2b", C.c_int32),
        ("een_cusp", C.c_int32),
        ("a4", C.POINTER(C.c_double)), ("b", C.POINTER(C.c_double)), ("c", C.POINTER(C.c_double)),
        ("nloc", C.c_int32), ("nquad", C.c_int32), ("mgauss", C.c_int32),
        ("npotd", C.POINTER(C.c_int32)), ("lpotp1", C.POINTER(C.c_int32)),
        ("necp_term", C.POINTER(C.c_int32)), ("necp_power", C.POINTER(C.c_int32)),
        ("ecp_coef", C.POINTER(C.c_double)), ("ecp_exponent", C.POINTER(C.c_double)),
        ("nrad", C.c_int32), ("rad_igrid", C.POINTER(C.c_int32)), ("rad_nr", C.POINTER(C.c_int32)),
        ("rad_h", C.POINTER(C.c_double)), ("rad_r0", C.POINTER(C.c_double)), ("rad_x", C.POINTER(C.c_double)),
        ("rad_val", C.POINTER(C.c_double)), ("shell_rad", C.POINTER(C.c_int32)),
    ]


def nterms4(nord: int) -> int:
    """Number of e-e-n terms of order <= nord (nterms4, qmc/vmc/jastrow4.f90:495)."""
    i = 0
    for n in range(2, nord + 1):
        for k in range(n - 1, -1, -1):
            l_hi = n - k - 2 if k == 0 else n - k
            for l in range(l_hi, -1, -1):
                m = (n - k - l) // 2
                if 2 * m == n - k - l:
                    i += 1
    return i


@dataclass
class System:
    name: str
    nelec: int
    nup: int
    cent: np.ndarray            # [ncent,3]
    iwctype: np.ndarray         # [ncent]
    znuc: np.ndarray            # [nctype]
    shell_cent: np.ndarray
    shell_n: np.ndarray
    shell_l: np.ndarray
    shell_kind: np.ndarray
    shell_nprim: np.ndarray
    prim_zeta: np.ndarray
    prim_coef: np.ndarray
    basis_shell: np.ndarray
    basis_m: np.ndarray
    coef: np.ndarray            # [norb, nbasis]
    det_orb: np.ndarray         # [ndet, nelec]
    csf_coef: np.ndarray
    csf_ndet: np.ndarray
    csf_det: np.ndarray
    csf_det_coef: np.ndarray
    scalek: float
    norda: int
    nordb: int
    nordc: int
    nspin2b: int
    een_cusp: int
    a4: np.ndarray              # [nctype, norda+1]
    b: np.ndarray               # [nspin2b, nordb+1]
    c: np.ndarray               # [nctype, nterms]
    nloc: int = 0
    nquad: int = 12
    npotd: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    lpotp1: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    necp_term: np.ndarray = field(default_factory=lambda: np.zeros((1, MAX_LCHAN), np.int32))
    necp_power: np.ndarray = field(default_factory=lambda: np.zeros((1, MAX_LCHAN, 1), np.int32))
    ecp_coef: np.ndarray = field(default_factory=lambda: np.zeros((1, MAX_LCHAN, 1)))
    ecp_exponent: np.ndarray = field(default_factory=lambda: np.zeros((1, MAX_LCHAN, 1)))
    # numerical radial tables (shell kind 2): grid type, points, step or ratio, r0 as read,
    # grid points and values of every table one after another, and each shell's table
    rad_igrid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    rad_nr: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    rad_h: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rad_r0: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rad_x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rad_val: np.ndarray = field(default_factory=lambda: np.zeros(0))
    shell_rad: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    walkers: int = 256          # walker count of the benchmark definition
    step: float = 0.5           # Metropolis step (bohr)

    @property
    def ncent(self):
        return len(self.cent)

    @property
    def nctype(self):
        return len(self.znuc)

    @property
    def nbasis(self):
        return len(self.basis_shell)

    @property
    def norb(self):
        return self.coef.shape[0]

    @property
    def ndet(self):
        return self.det_orb.shape[0]

    def to_c(self):
        """Pack into a ChampSystem; returns (struct, keepalive)."""
        keep = []

        def P(arr, dt):
            a = np.ascontiguousarray(arr, dtype=dt)
            keep.append(a)
            ct = C.c_double if dt == np.float64 else C.c_int32
            return a.ctypes.data_as(C.POINTER(ct))

        f8, i4 = np.float64, np.int32
        mg = max(1, self.ecp_coef.shape[-1])
        s = ChampSystem(
            nelec=self.nelec, nup=self.nup, ncent=self.ncent, nctype=self.nctype,
            cent=P(self.cent, f8), iwctype=P(self.iwctype, i4), znuc=P(self.znuc, f8),
            nshell=len(self.shell_cent),
            shell_cent=P(self.shell_cent, i4), shell_n=P(self.shell_n, i4), shell_l=P(self.shell_l, i4),
            shell_kind=P(self.shell_kind, i4), shell_nprim=P(self.shell_nprim, i4),
            prim_zeta=P(self.prim_zeta, f8), prim_coef=P(self.prim_coef, f8),
            nbasis=self.nbasis, basis_shell=P(self.basis_shell, i4), basis_m=P(self.basis_m, i4),
            norb=self.norb, coef=P(self.coef, f8),
            ndet=self.ndet, det_orb=P(self.det_orb, i4),
            ncsf=len(self.csf_coef), csf_coef=P(self.csf_coef, f8), csf_ndet=P(self.csf_ndet, i4),
            csf_det=P(self.csf_det, i4), csf_det_coef=P(self.csf_det_coef, f8),
            scalek=self.scalek, norda=self.norda, nordb=self.nordb, nordc=self.nordc,
            nspin2b=self.nspin2b, een_cusp=self.een_cusp,
            a4=P(self.a4, f8), b=P(self.b, f8), c=P(self.c if self.c.size else np.zeros(1), f8),
            nloc=self.nloc, nquad=self.nquad, mgauss=mg,
            npotd=P(self.npotd, i4), lpotp1=P(self.lpotp1, i4),
            necp_term=P(self.necp_term, i4), necp_power=P(self.necp_power, i4),
            ecp_coef=P(self.ecp_coef, f8), ecp_exponent=P(self.ecp_exponent, f8),
            nrad=len(self.rad_igrid), rad_igrid=P(np.append(self.rad_igrid, 0), i4),
            rad_nr=P(np.append(self.rad_nr, 0), i4), rad_h=P(np.append(self.rad_h, 0.0), f8),
            rad_r0=P(np.append(self.rad_r0, 0.0), f8), rad_x=P(np.append(self.rad_x, 0.0), f8),
            rad_val=P(np.append(self.rad_val, 0.0), f8),
            shell_rad=P(self.shell_rad if len(self.shell_rad) else np.full(len(self.shell_cent), -1), i4),
        )
        return s, keep


# --------------------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------------------
_M_ORDER = {0: [0], 1: [1, -1, 0], 2: [0, 1, -1, 2, -2], 3: [0, 1, -1, 2, -2, 3, -3],
            4: [0, 1, -1, 2, -2, 3, -3, 4, -4]}


def _basis_from_shells(shells):
    """shells: list of (centre, n, l, kind, zetas, coefs) -> shell and basis arrays."""
    sc, sn, sl, sk, snp, pz, pc, bs, bm = [], [], [], [], [], [], [], [], []
    for ish, (cen, n, l, kind, z, w) in enumerate(shells):
        sc.append(cen); sn.append(n); sl.append(l); sk.append(kind); snp.append(len(z))
        pz.extend(z); pc.extend(w)
        for m in _M_ORDER[l]:
            bs.append(ish); bm.append(m)
    i4 = np.int32
    return dict(shell_cent=np.array(sc, i4), shell_n=np.array(sn, i4), shell_l=np.array(sl, i4),
                shell_kind=np.array(sk, i4), shell_nprim=np.array(snp, i4),
                prim_zeta=np.array(pz, float), prim_coef=np.array(pc, float),
                basis_shell=np.array(bs, i4), basis_m=np.array(bm, i4))


def _orthonormal_rows(rng, nrow, ncol):
    """Random N(0,1) rows, Gram-Schmidt orthonormalised (as a QR factorisation)."""
    a = rng.standard_normal((ncol, nrow))
    q, r = np.linalg.qr(a)
    q = q * np.sign(np.diag(r))[None, :]
    return np.ascontiguousarray(q.T)


def _single_det(nelec, nup):
    ndn = nelec - nup
    row = list(range(nup)) + list(range(ndn))
    return np.array([row], np.int32)


def _one_csf(ndet=1):
    return dict(csf_coef=np.ones(1), csf_ndet=np.array([1], np.int32),
                csf_det=np.zeros(1, np.int32), csf_det_coef=np.ones(1))


def _gaussian_ecp(rng, nctype):
    """s and p channels, 2 Gaussian terms each; p (channel 2) local as in the C2 example."""
    ecp_coef = np.zeros((nctype, MAX_LCHAN, 2))
    ecp_exp = np.zeros((nctype, MAX_LCHAN, 2))
    ecp_pow = np.zeros((nctype, MAX_LCHAN, 2), np.int32)
    necp = np.zeros((nctype, MAX_LCHAN), np.int32)
    for it in range(nctype):
        for l in range(2):
            necp[it, l] = 2
            ecp_exp[it, l] = rng.uniform(0.5, 10.0, 2)
            ecp_coef[it, l] = rng.uniform(-5.0, 5.0, 2)
            ecp_pow[it, l] = 2
    return dict(nloc=6, nquad=12, npotd=np.full(nctype, 2, np.int32), lpotp1=np.full(nctype, 2, np.int32),
                necp_term=necp, necp_power=ecp_pow, ecp_coef=ecp_coef, ecp_exponent=ecp_exp)


def _jastrow(rng, nctype, norda=5, nordb=5, nordc=0, c_scale=0.02):
    a4 = np.zeros((nctype, norda + 1))
    for it in range(nctype):
        a4[it, 2:] = rng.uniform(-0.1, 0.1, norda - 1)
    b = np.zeros((1, nordb + 1))
    b[0, 0] = 0.5
    b[0, 1] = 1.0
    b[0, 2:] = rng.uniform(-0.1, 0.1, nordb - 1)
    nt = nterms4(nordc)
    c = rng.uniform(-c_scale, c_scale, (nctype, nt)) if nt else np.zeros((nctype, 0))
    return dict(scalek=0.8, norda=norda, nordb=nordb, nordc=nordc, nspin2b=1, een_cusp=1 if nt else 0,
                a4=a4, b=b, c=c)


def _contracted_gaussian_shells(rng, ncent, per_centre, nprim=3):
    """per_centre: list of (n, l).  Exponents log-uniform in [0.1, 30], weights N(0,1)."""
    shells = []
    for ic in range(ncent):
        for (n, l) in per_centre:
            z = np.exp(rng.uniform(np.log(0.1), np.log(30.0), nprim))
            w = rng.standard_normal(nprim)
            shells.append((ic, n, l, 1, list(z), list(w)))
    return shells


# --------------------------------------------------------------------------------------
# the five benchmark systems
# --------------------------------------------------------------------------------------
def be_atom(seed=1001) -> System:
    """System 1: all-electron Be-like atom, Slater basis 1s(3.5,6.0) 2s(0.9,1.6) 2p(1.0)."""
    rng = np.random.default_rng(seed)
    r_orb, r_jas = [np.random.default_rng(s) for s in rng.integers(0, 2**63, 2)]
    shells = [(0, 1, 0, 0, [3.5], [1.0]), (0, 1, 0, 0, [6.0], [1.0]),
              (0, 2, 0, 0, [0.9], [1.0]), (0, 2, 0, 0, [1.6], [1.0]),
              (0, 2, 1, 0, [1.0], [1.0])]
    bas = _basis_from_shells(shells)
    nb = len(bas["basis_shell"])
    coef = _orthonormal_rows(r_orb, nb, nb)
    return System(name="be_atom", nelec=4, nup=2, cent=np.zeros((1, 3)), iwctype=np.zeros(1, np.int32),
                  znuc=np.array([4.0]), **bas, coef=coef, det_orb=_single_det(4, 2), **_one_csf(),
                  **_jastrow(r_jas, 1, 5, 5, 0), walkers=256, step=0.5)


def c2_dimer(seed=1002, nordc=4, norb=16) -> System:
    """System 2: C2-like pseudopotential dimer, 60 contracted Gaussians, 1 determinant; norb
    orthonormal orbitals (the determinants use the first 16)."""
    rng = np.random.default_rng(seed)
    r_bas, r_orb, r_jas, r_ecp = [np.random.default_rng(s) for s in rng.integers(0, 2**63, 4)]
    per_centre = [(1, 0)] * 6 + [(2, 1)] * 3 + [(3, 2)] * 3
    bas = _basis_from_shells(_contracted_gaussian_shells(r_bas, 2, per_centre))
    nb = len(bas["basis_shell"])
    coef = _orthonormal_rows(r_orb, norb, nb)
    cent = np.array([[0.0, 0.0, 1.175], [0.0, 0.0, -1.175]])
    return System(name="c2_dimer", nelec=8, nup=4, cent=cent, iwctype=np.zeros(2, np.int32),
                  znuc=np.array([4.0]), **bas, coef=coef, det_orb=_single_det(8, 4), **_one_csf(),
                  **_jastrow(r_jas, 1, 5, 5, nordc), **_gaussian_ecp(r_ecp, 1), walkers=8192, step=0.5)


def c2_multidet(seed=1003, ndet=200, ncsf=60, norb_act=16, norb=36) -> System:
    """System 3: system 2 with ndet seeded single/double excitations in 16 orbitals, grouped
    into ncsf CSFs whose coefficients decay as 0.5**(excitation rank); 36 orbitals, so that the
    optimisable parameters (59 CSF, 440 orbital rotations: 120 among the 16 active orbitals and
    16 x 20 active -> virtual, 16 Jastrow) number 515."""
    base = c2_dimer(norb=norb)
    rng = np.random.default_rng(seed)
    nup = ndn = 4
    ref = tuple(range(nup)), tuple(range(ndn))
    dets = {ref: 0}
    order = [ref]
    ranks = [0]
    while len(order) < ndet:
        kind = rng.integers(0, 5)  # 0: up single, 1: dn single, 2: up-dn double, 3: up-up, 4: dn-dn
        up, dn = list(ref[0]), list(ref[1])

        def excite(lst, nh):
            holes = rng.choice(len(lst), nh, replace=False)
            parts = rng.choice(np.arange(len(lst), norb_act), nh, replace=False)
            for h, p in zip(holes, parts):
                lst[h] = int(p)
        if kind == 0: excite(up, 1); rk = 1
        elif kind == 1: excite(dn, 1); rk = 1
        elif kind == 2: excite(up, 1); excite(dn, 1); rk = 2
        elif kind == 3: excite(up, 2); rk = 2
        else: excite(dn, 2); rk = 2
        key = (tuple(up), tuple(dn))
        if key in dets:
            continue
        dets[key] = len(order)
        order.append(key)
        ranks.append(rk)
    det_orb = np.array([list(u) + list(d) for (u, d) in order], np.int32)
    # CSF 0 = reference; the others get consecutive groups of excited determinants
    groups = np.array_split(np.arange(1, ndet), ncsf - 1)
    csf_ndet = [1] + [len(g) for g in groups]
    csf_det = [0] + [int(i) for g in groups for i in g]
    csf_det_coef = [1.0] + list(rng.choice([-1.0, 1.0], ndet - 1))
    csf_coef = [1.0] + [float(rng.choice([-1.0, 1.0]) * 0.5 ** max(ranks[g[0]] for _ in [0]) * rng.uniform(0.2, 1.0))
                        for g in groups]
    base.name = "c2_multidet"
    base.det_orb = det_orb
    base.csf_coef = np.array(csf_coef)
    base.csf_ndet = np.array(csf_ndet, np.int32)
    base.csf_det = np.array(csf_det, np.int32)
    base.csf_det_coef = np.array(csf_det_coef)
    base.walkers = 16384
    return base


def c2_dmc(seed=1004) -> System:
    """System 4: system 2 (single determinant) for DMC with a target population of 32768."""
    s = c2_dimer()
    s.name = "c2_dmc"
    s.walkers = 32768
    return s


def cluster128(seed=1005, ncent=32, box=14.0, dmin=2.5, norb=96) -> System:
    """System 5: 32 pseudo-atoms (Z_eff=4) uniform in a 14-bohr cube with minimum separation
    2.5 bohr, 64+64 electrons, 13 contracted Gaussians per centre (2s 2p 1d)."""
    rng = np.random.default_rng(seed)
    r_geo, r_bas, r_orb, r_jas, r_ecp = [np.random.default_rng(s) for s in rng.integers(0, 2**63, 5)]
    cent = []
    while len(cent) < ncent:
        p = r_geo.uniform(0.0, box, 3)
        if all(np.linalg.norm(p - q) >= dmin for q in cent):
            cent.append(p)
    cent = np.array(cent) - box / 2
    per_centre = [(1, 0), (1, 0), (2, 1), (2, 1), (3, 2)]
    bas = _basis_from_shells(_contracted_gaussian_shells(r_bas, ncent, per_centre))
    nb = len(bas["basis_shell"])
    coef = _orthonormal_rows(r_orb, norb, nb)
    return System(name="cluster128", nelec=128, nup=64, cent=cent, iwctype=np.zeros(ncent, np.int32),
                  znuc=np.array([4.0]), **bas, coef=coef, det_orb=_single_det(128, 64), **_one_csf(),
                  **_jastrow(r_jas, 1, 5, 5, 4), **_gaussian_ecp(r_ecp, 1), walkers=4096, step=0.3)


SYSTEMS = {1: be_atom, 2: c2_dimer, 3: c2_multidet, 4: c2_dmc, 5: cluster128}


def get_system(k: int) -> System:
    return SYSTEMS[k]()


def initial_walkers(sys: System, nw: int, seed: int = 7, mean_radius: float = 1.5) -> np.ndarray:
    """Electron starts: radius ~ Exp(mean 1.5 bohr), isotropic direction, around the centres
    in turn.  Returns x[nw, nelec, 3]."""
    rng = np.random.default_rng(seed)
    ne = sys.nelec
    r = rng.exponential(mean_radius, (nw, ne))
    v = rng.standard_normal((nw, ne, 3))
    v /= np.linalg.norm(v, axis=2, keepdims=True)
    cidx = np.arange(ne) % sys.ncent
    # spread each spin over the centres
    cidx = np.concatenate([np.arange(sys.nup) % sys.ncent, np.arange(ne - sys.nup) % sys.ncent])
    x = sys.cent[cidx][None, :, :] + r[..., None] * v
    return np.ascontiguousarray(x)


def from_slater_example(fx: dict) -> System:
    """Builds a System from a parsed CHAMP keyword input with an analytic Slater basis
    on one centre (the dictionary written by tests/golden/make_be_fixture.py):
    basis names like 1S, 2S, 2PX, 2PY, 2PZ with exponents, orbital coefficients,
    determinants (1-based orbitals), CSFs and ijas=4 Jastrow parameters."""
    lmap = {"S": 0, "P": 1}
    mmap = {"S": 0, "PX": 1, "PY": -1, "PZ": 0}
    shells, bshell, bm = [], [], []
    key = {}
    for name, z in fx["basis"]:
        n = int(name[0]); ang = name[1:]
        l = lmap[ang[0]]
        k = (n, l, z)
        if l == 0 or k not in key:
            key[k] = len(shells)
            shells.append((0, n, l, 0, [z], [1.0]))
        bshell.append(key[k]); bm.append(mmap[ang])
    bas = _basis_from_shells(shells)
    # keep the input's basis-function order
    bas["basis_shell"] = np.array(bshell, np.int32)
    bas["basis_m"] = np.array(bm, np.int32)
    order = np.argsort(np.array(bshell), kind="stable")
    assert np.all(np.diff(np.array(bshell)[order]) >= 0)
    coef = np.array(fx["coef"], float)
    ne, nup = fx["nelec"], fx["nup"]
    det_orb = np.array(fx["dets"], np.int32) - 1
    ncsf = len(fx["csf_coef"])
    csf_det = [d - 1 for ds in fx["csf_dets"] for d in ds]
    csf_cdet = [c for cs in fx["csf_cdet"] for c in cs]
    a = np.array(fx["a"], float)[None, :]
    b = np.array(fx["b"], float)[None, :]
    c = np.array(fx["c"], float)[None, :]
    nord_a, nord_b = a.shape[1] - 1, b.shape[1] - 1
    nordc = 0
    while nterms4(nordc + 1) <= c.shape[1] and nordc < 7:
        nordc += 1
    return System(name="be_example", nelec=ne, nup=nup, cent=np.zeros((1, 3)), iwctype=np.zeros(1, np.int32),
                  znuc=np.array([fx["znuc"]]), **bas, coef=coef, det_orb=det_orb,
                  csf_coef=np.array(fx["csf_coef"], float), csf_ndet=np.array([len(d) for d in fx["csf_dets"]], np.int32),
                  csf_det=np.array(csf_det, np.int32), csf_det_coef=np.array(csf_cdet, float),
                  scalek=fx["scalek"], norda=nord_a, nordb=nord_b, nordc=nordc, nspin2b=1, een_cusp=0,
                  a4=a, b=b, c=c, walkers=1024, step=0.5)


def be_example() -> System:
    """The reference's Be example wave function (fixture tests/golden/be_vb1.json)."""
    import json
    import os
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(here, "tests", "golden", "be_vb1.json")) as f:
        return from_slater_example(json.load(f))


_LABEL_LM = {"S": (0, 0), "PX": (1, 1), "PY": (1, -1), "PZ": (1, 0)}
for _l, _c in ((2, "D"), (3, "F"), (4, "G")):
    _LABEL_LM[f"{_c}0"] = (_l, 0)
    for _m in range(1, _l + 1):
        _LABEL_LM[f"{_c}+{_m}"] = (_l, _m)
        _LABEL_LM[f"{_c}-{_m}"] = (_l, -_m)


def c2_bfd_fixture():
    """The parsed reference example (tests/golden/c2_bfd.npz, made by make_c2_bfd_fixture.py)."""
    import json
    import os
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    d = np.load(os.path.join(here, "tests", "golden", "c2_bfd.npz"))
    return json.loads(str(d["meta"])), d["coef"], d["grid_x"], d["grid_val"]


def c2_bfd_example(run: int = 0) -> System:
    """The reference's C2 pseudopotential example (examples/c2_bfd_vtz_rhf_vmc_new.inp): two
    carbon pseudo-atoms (Z_eff 4), 68 basis functions on 9 numerical radial functions
    (examples/basis.1, splined as splfit_bas does), BFD pseudopotential with an s nonlocal
    channel (examples/pseudopot1), 6-point quadrature, one determinant, Jastrow ijas=4 isc=4
    with the parameters of VMC run `run` of the transcript (0: the input's)."""
    meta, coef, gx, gv = c2_bfd_fixture()
    par = meta["runs"][run]["params"]
    shells, bshell, bm, srad, key = [], [], [], [], {}
    ncent = len(meta["cent"])
    for ic in range(ncent):
        for lab, irad in meta["labels"]:
            l, m = _LABEL_LM[lab.upper()]
            k = (ic, l, irad)
            if k not in key:
                key[k] = len(shells)
                shells.append((ic, l + 1, l, 2, [0.0], [1.0]))
                srad.append(irad - 1)
            bshell.append(key[k])
            bm.append(m)
    bas = _basis_from_shells(shells)
    bas["basis_shell"] = np.array(bshell, np.int32)
    bas["basis_m"] = np.array(bm, np.int32)
    g = meta["grid"]
    nrb = g["nrbas"]
    ps = meta["pseudopot"]
    nct = len(meta["znuc"])
    necp = np.zeros((nct, MAX_LCHAN), np.int32)
    mg = max(len(t) for t in ps["components"])
    ecoef, eexp = np.zeros((nct, MAX_LCHAN, mg)), np.zeros((nct, MAX_LCHAN, mg))
    epow = np.zeros((nct, MAX_LCHAN, mg), np.int32)
    lpotp1 = meta["lpotp1"]
    for it in range(nct):
        for k, terms in enumerate(ps["components"]):
            ch = lpotp1[it] - 1 if k == 0 else k - 1  # local component first in the file
            necp[it, ch] = len(terms)
            for i, (cf, pw, ex) in enumerate(terms):
                ecoef[it, ch, i], epow[it, ch, i], eexp[it, ch, i] = cf, pw, ex
    a = np.array(par["a"], float)[None, :]
    b = np.array(par["b"], float)[None, :]
    c = np.array(par["c"], float)[None, :]
    nordc = 0
    while nterms4(nordc + 1) <= c.shape[1] and nordc < 7:
        nordc += 1
    ne, nup = meta["nelec"], meta["nup"]
    det = np.array(meta["iworbd"], np.int32)[None, :] - 1
    return System(name="c2_bfd_example", nelec=ne, nup=nup, cent=np.array(meta["cent"], float),
                  iwctype=np.array(meta["iwctype"], np.int32), znuc=np.array(meta["znuc"], float), **bas,
                  coef=np.ascontiguousarray(coef), det_orb=det, **_one_csf(), scalek=meta["scalek"],
                  norda=a.shape[1] - 1, nordb=b.shape[1] - 1, nordc=nordc, nspin2b=1, een_cusp=1 if nordc > 1 else 0,
                  a4=a, b=b, c=c, nloc=meta["nloc"], nquad=meta["nquad"], npotd=np.full(nct, ps["npotd"], np.int32),
                  lpotp1=np.array(lpotp1, np.int32), necp_term=necp, necp_power=epow, ecp_coef=ecoef,
                  ecp_exponent=eexp, rad_igrid=np.full(nrb, g["igrid"], np.int32), rad_nr=np.full(nrb, g["nr"], np.int32),
                  rad_h=np.full(nrb, g["exph"]), rad_r0=np.full(nrb, g["r0"]), rad_x=np.tile(gx, nrb),
                  rad_val=np.ascontiguousarray(gv).ravel(), shell_rad=np.array(srad, np.int32), walkers=8192,
                  step=0.45)


def hydrogenic(z=2.0) -> System:
    """One electron in a Slater 1s orbital of exponent z around charge z, no Jastrow:
    the exact eigenfunction, E_L = -z^2/2 everywhere."""
    bas = _basis_from_shells([(0, 1, 0, 0, [z], [1.0])])
    return System(name="hydrogenic", nelec=1, nup=1, cent=np.zeros((1, 3)), iwctype=np.zeros(1, np.int32),
                  znuc=np.array([z]), **bas, coef=np.ones((1, 1)), det_orb=np.zeros((1, 1), np.int32), **_one_csf(),
                  scalek=0.8, norda=5, nordb=5, nordc=0, nspin2b=1, een_cusp=0,
                  a4=np.zeros((1, 6)), b=np.zeros((1, 6)), c=np.zeros((1, 0)))
