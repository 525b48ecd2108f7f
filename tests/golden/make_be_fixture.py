"""Generates tests/golden/be_vb1.json from the reference's Be example.

Reads the CHAMP example input examples/be_vb1_jcas24_vmc_j_opt_lin.inp (Be atom, Slater
basis, 4 determinants in 4 CSFs, ijas=4/isc=4 Jastrow with only b1=0.5, b2=1) and the
first 'Final results' block of its transcript examples/be_vb1_jcas24_vmc_j_opt_lin.out
(the VMC run with the input parameters, before any optimisation step).  The JSON keeps
the parsed wave function and the reference's printed averages, so that the VMC energy
of this wave function can be compared with the reference's without the reference tree.

Usage: python tests/golden/make_be_fixture.py /path/to/CHAMP
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_be_fixture.py /path/to/CHAMP")
ROOT = sys.argv[1]
INP = os.path.join(ROOT, "examples", "be_vb1_jcas24_vmc_j_opt_lin.inp")
OUT = os.path.join(ROOT, "examples", "be_vb1_jcas24_vmc_j_opt_lin.out")


def block(text, name):
    m = re.search(r"^\s*%s\s*$(.*?)^\s*end\s*$" % name, text, re.S | re.M)
    return m.group(1)


def main():
    txt = open(INP).read()
    bas = block(txt, "basis_functions").split("\n")
    bas = [l.split() for l in bas if l.strip()]
    ctype_count = int(bas[0][0])
    funcs = [(b[0], float(b[1])) for b in bas[1:]]
    coef = [[float(v) for v in l.split()[:8]] for l in block(txt, "coefficients").split("\n")
            if l.strip() and not l.strip().startswith("(")]
    dets = [[int(v) for v in l.split()[:4]] for l in block(txt, "determinants").split("\n") if l.strip()]
    csf_line = re.search(r"csf_coef(.*?)end", txt).group(1)
    csf_coef = [float(v) for v in csf_line.split()]
    dic = [l.split() for l in block(txt, "dets_in_csfs").split("\n") if l.strip()]
    csf_dets = [[int(v) for v in dic[2 * i]] for i in range(len(csf_coef))]
    csf_cdet = [[float(v) for v in dic[2 * i + 1]] for i in range(len(csf_coef))]
    jb = [l.split("(")[0].split() for l in block(txt, "parameters").split("\n") if l.strip()]
    a = [float(v) for v in jb[0]]
    b = [float(v) for v in jb[1]]
    c = [float(v) for v in jb[2]]
    scalek = float(re.search(r"scalek\s*=\s*([0-9.]+)", txt).group(1))
    out = open(OUT).read()
    fr = out.index("Final results after")
    seg = out[fr:fr + 2000]
    def grab(label):
        m = re.search(label + r"\s*=\s*([-0-9.]+)\s*\+-\s*([0-9.]+)", seg)
        return float(m.group(1)), float(m.group(2))
    E, dE = grab("total E")
    PE, dPE = grab("potential E")
    R2, dR2 = grab("<r2>")
    sig = float(re.search(r"total E\s*=\s*[-0-9.]+\s*\+-\s*[0-9.]+\s+[0-9.]+\s+([0-9.]+)", seg).group(1))
    passes = int(float(re.search(r"Final results after\s+([0-9.]+)\s*passes", seg).group(1)))
    fix = dict(source=dict(input="examples/be_vb1_jcas24_vmc_j_opt_lin.inp",
                           transcript="examples/be_vb1_jcas24_vmc_j_opt_lin.out"),
               nctype_line=ctype_count, basis=funcs, coef=coef, dets=dets, csf_coef=csf_coef,
               csf_dets=csf_dets, csf_cdet=csf_cdet, a=a, b=b, c=c, scalek=scalek, znuc=4.0, nelec=4, nup=2,
               reference=dict(energy=E, energy_err=dE, sigma=sig, pe=PE, pe_err=dPE, r2=R2, r2_err=dR2,
                              passes=passes))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "be_vb1.json")
    json.dump(fix, open(dst, "w"), indent=1)
    print(dst, fix["reference"])


if __name__ == "__main__":
    main()
