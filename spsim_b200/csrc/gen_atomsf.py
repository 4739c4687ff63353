"""Regenerate ``atomsf_data.h``: the 4-Gaussian + constant X-ray form-factor
coefficients (a1..a4, b1..b4, c) for Z = 0..99.

The numbers are CCP4's ``atomsf.lib`` values (International Tables for
Crystallography Vol. C, Table 6.1.1.4), the same table spsim compiles in from
``include/atomsf.cdata`` and indexes by atomic number (row Z; row 0 and row 99
are the table's ``-1`` placeholders).  Structure-factor parity needs the
identical coefficients, so this script reads that table once and writes it out
in this project's own layout.  It is a maintenance tool; nothing at build or
run time calls it.

Usage: python gen_atomsf.py <path-to-atomsf.cdata> > atomsf_data.h
"""
import re
import sys

SYMBOLS = (
    "X H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni "
    "Cu Zn Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe "
    "Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg "
    "Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es"
).split()


def main(path):
    text = open(path).read()
    rows = re.findall(r"\{([^{}]*)\}", text)
    table = [[float(v) for v in r.split(",")] for r in rows]
    assert len(table) == 100 and all(len(r) == 9 for r in table), "unexpected table shape"
    out = [
        "/* Generated by gen_atomsf.py: X-ray form-factor coefficients f0(s) =",
        " * sum_i a_i exp(-b_i s^2) + c with s = |q|/2 in 1/Angstrom, for Z = 0..99",
        " * (CCP4 atomsf.lib / International Tables Vol. C 6.1.1.4).  Rows 0 and 99",
        " * are placeholders {a1=-1, rest 0}, as in the table spsim ships. */",
        "#ifndef SPSIM_B200_ATOMSF_DATA_H",
        "#define SPSIM_B200_ATOMSF_DATA_H",
        "#define SPSIM_B200_N_ELEMENTS 100",
        "/* per row: a1 a2 a3 a4 b1 b2 b3 b4 c */",
        "static const float spsim_b200_atomsf_default[SPSIM_B200_N_ELEMENTS][9] = {",
    ]
    for z, r in enumerate(table):
        sym = SYMBOLS[z] if z < len(SYMBOLS) else "-"
        vals = ", ".join("%.6ef" % v for v in r)
        out.append("  /* %2d %-2s */ {%s}," % (z, sym, vals))
    out += ["};", "#endif", ""]
    sys.stdout.write("\n".join(out))


if __name__ == "__main__":
    main(sys.argv[1])
