"""Builds tests/golden/c2_bfd.npz from the reference's C2 pseudopotential example.

Reads, from the reference tree given on the command line (the directory holding ``examples/``):
  examples/c2_bfd_vtz_rhf_vmc_new.inp   nuclei, basis labels, orbitals, determinant, Jastrow
  examples/basis.1                      numerical radial basis on a grid (read_bas_num.f90)
  examples/pseudopot1                   Gaussian pseudopotential (readps_gauss.f90 format)
  examples/c2_bfd_vtz_rhf_vmc_new.out   the VMC energies of the transcript and, for each run,
                                        the Jastrow parameters it was run with (the input's,
                                        then each "New wave function" of the optimisation)

Usage: python tests/golden/make_c2_bfd_fixture.py <reference-root>
The fixture is consumed by champ_b200.system.c2_bfd_example() and the tests; nothing at run
time reads the reference tree.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[EeDd][-+]?\d+)?"


def _floats(line):
    return [float(t.replace("D", "E").replace("d", "e")) for t in re.findall(NUM, line)]


def _block(lines, name):
    """Lines between '<name>' and its 'end' (top-level keyword blocks open and close in column 0;
    their sub-blocks close with an indented ' end')."""
    out, on = [], False
    for ln in lines:
        if not on:
            if ln.strip() == name and not ln.startswith(" "):
                on = True
            continue
        if ln.rstrip() == "end":
            return out
        out.append(ln)
    raise ValueError(f"block {name} not found")


def _sub(block, name):
    """Lines of a sub-block ' name' ... ' end' inside a block."""
    out, on = [], False
    for ln in block:
        t = ln.strip()
        if not on:
            if t.split() and t.split()[0] == name:
                on = True
            continue
        if t == "end":
            return out
        out.append(ln)
    raise ValueError(f"sub-block {name} not found")


def parse_input(path):
    lines = open(path).read().splitlines()
    nuc = _block(lines, "nuclei")
    geo = _sub(nuc, "geometry")
    cent, iwctype, znuc = [], [], {}
    for ln in geo:
        f = ln.split()
        it = int(f[0])
        znuc[it] = float(f[1])
        iwctype.append(it - 1)
        cent.append([float(v) for v in f[2:5]])
    kv = " ".join(nuc)
    nloc = int(re.search(r"nloc\s*=\s*(\d+)", kv).group(1))
    nquad = int(re.search(r"nquad\s*=\s*(\d+)", kv).group(1))
    lpotp1 = [int(v) for v in re.search(r"lpotp1\s+([\d\s]+)\s+end", kv).group(1).split()]
    wf = " ".join(_block(lines, "wavefunction"))
    nelec = int(re.search(r"nelec\s*=\s*(\d+)", wf).group(1))
    nup = int(re.search(r"nup\s*=\s*(\d+)", wf).group(1))
    bas = _sub(_block(lines, "basis"), "basis_functions")
    nctype_bas = int(bas[0].split()[0])
    labels = [(ln.split()[0], int(ln.split()[1])) for ln in bas[1:] if ln.strip()]
    orb = _sub(_block(lines, "orbitals"), "coefficients")
    coef = [_floats(ln.split("(")[0]) for ln in orb if ln.strip()]
    nb = len(coef[0])
    coef = np.array([c[:nb] for c in coef])
    dets = _sub(_block(lines, "csfs"), "determinants")
    iworbd = [int(v) for v in dets[0].split("(")[0].split()]
    jas = _block(lines, "jastrow")
    jkv = " ".join(jas)
    scalek = float(re.search(r"scalek\s*=\s*(" + NUM + ")", jkv).group(1))
    par = _sub(jas, "parameters")
    a = _floats(par[0].split("(")[0])
    b = _floats(par[1].split("(")[0])
    c = _floats(par[2].split("(")[0])
    return dict(cent=cent, iwctype=iwctype, znuc=[znuc[k] for k in sorted(znuc)], nloc=nloc, nquad=nquad,
                lpotp1=lpotp1, nelec=nelec, nup=nup, nctype_bas=nctype_bas, labels=labels, coef=coef,
                iworbd=iworbd, scalek=scalek, a=a, b=b, c=c)


def parse_basis1(path):
    """basis.1 (read_bas_num.f90): comment lines start with '#'; then
    'nrbas igrid nr exp_h_bas r0_bas icusp', then nr rows of r and the nrbas radial values."""
    rows = [ln for ln in open(path).read().splitlines() if ln.strip() and not ln.lstrip().startswith("#")]
    h = rows[0].split()
    nrbas, igrid, nr = int(h[0]), int(h[1]), int(h[2])
    exph, r0, icusp = float(h[3]), float(h[4]), int(h[5])
    data = np.array([_floats(r) for r in rows[1:1 + nr]])
    assert data.shape == (nr, nrbas + 1), data.shape
    return dict(nrbas=nrbas, igrid=igrid, nr=nr, exph=exph, r0=r0, icusp=icusp, x=data[:, 0],
                val=np.ascontiguousarray(data[:, 1:].T))


def parse_pseudopot(path):
    """readps_gauss.f90: label; number of components; per component (local first): number of
    terms, then 'coefficient power exponent' per term."""
    toks = open(path).read().split("\n")
    label = toks[0].strip()
    rest = " ".join(toks[1:]).split()
    i = 0
    npotd = int(rest[i]); i += 1
    comps = []
    for _ in range(npotd):
        nt = int(rest[i]); i += 1
        terms = []
        for _ in range(nt):
            terms.append((float(rest[i]), int(rest[i + 1]), float(rest[i + 2])))
            i += 3
        comps.append(terms)
    return dict(label=label, npotd=npotd, components=comps)


def parse_transcript(path, params0):
    """Every single-wave-function VMC result ('Final results' followed by 'total E =') with the
    Jastrow parameters in effect: the input's, replaced after each 'New wave function:'."""
    lines = open(path).read().splitlines()
    cur = dict(a=list(params0["a"]), b=list(params0["b"]), c=list(params0["c"]))
    runs = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("New wave function:"):
            new = {}
            for j in range(i + 1, min(i + 8, len(lines))):
                for key in ("a", "b", "c"):
                    if f"({key}_new(iparmj)" in lines[j]:
                        new[key] = _floats(lines[j].split("(")[0])
            assert set(new) == {"a", "b", "c"}, new
            cur = new
        m = re.match(r"Final results after\s+(" + NUM + r")\s+passes", ln)
        if m and i + 2 < len(lines) and lines[i + 2].startswith("total E ="):
            rec = {"passes": float(m.group(1)), "params": {k: list(v) for k, v in cur.items()}}
            for j in range(i + 2, i + 8):
                f = _floats(lines[j].split("=")[1]) if "=" in lines[j] else None
                if lines[j].startswith("total E ="):
                    rec["energy"], rec["energy_err"], rec["sigma"] = f[0], f[1], f[4]
                elif lines[j].startswith("potential E ="):
                    rec["pe"], rec["pe_err"] = f[0], f[1]
                elif lines[j].startswith("interaction E ="):
                    rec["pe_ee"], rec["pe_ee_err"] = f[0], f[1]
                elif lines[j].startswith("pb kinetic E ="):
                    rec["ke_pb"], rec["ke_pb_err"] = f[0], f[1]
            runs.append(rec)
        i += 1
    return runs


def main(root):
    ex = os.path.join(root, "examples")
    inp = parse_input(os.path.join(ex, "c2_bfd_vtz_rhf_vmc_new.inp"))
    b1 = parse_basis1(os.path.join(ex, "basis.1"))
    ps = parse_pseudopot(os.path.join(ex, "pseudopot1"))
    runs = parse_transcript(os.path.join(ex, "c2_bfd_vtz_rhf_vmc_new.out"), inp)
    meta = dict(source="examples/c2_bfd_vtz_rhf_vmc_new.inp, basis.1, pseudopot1, c2_bfd_vtz_rhf_vmc_new.out",
                nelec=inp["nelec"], nup=inp["nup"], nloc=inp["nloc"], nquad=inp["nquad"], lpotp1=inp["lpotp1"],
                cent=inp["cent"], iwctype=inp["iwctype"], znuc=inp["znuc"], labels=inp["labels"],
                iworbd=inp["iworbd"], scalek=inp["scalek"], a=inp["a"], b=inp["b"], c=inp["c"],
                grid=dict(nrbas=b1["nrbas"], igrid=b1["igrid"], nr=b1["nr"], exph=b1["exph"], r0=b1["r0"],
                          icusp=b1["icusp"]),
                pseudopot=ps, runs=runs)
    out = os.path.join(HERE, "c2_bfd.npz")
    np.savez_compressed(out, meta=np.array(json.dumps(meta)), coef=inp["coef"], grid_x=b1["x"], grid_val=b1["val"])
    print(out, "runs:", [(r["passes"], r["energy"], r["energy_err"]) for r in runs])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
