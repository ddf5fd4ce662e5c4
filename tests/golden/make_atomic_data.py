"""Writes tests/golden/atomic_data.npz: the reference's own atomic data tables,
parsed once in a container that holds the reference, so that the GPU tests and
the opacity benchmark run on the real tables where the reference is absent.

Sources (the reference's Data/ directory, SuperLite, GPLv3):

* ``data.bf_verner``: Verner et al. 1996 (ApJ 465, 487) and Verner & Yakovlev
  1995 (A&AS 109, 125) photo-ionisation fits, read as bfxs_read_data does
  (bfxsmod.f:144-180) into bf_ph1(6,7,30,30) and bf_ph2(7,30,30), real*4;
* ``data.ff_sutherland``: Sutherland 1998 (MNRAS 300, 321) free-free Gaunt
  factors, read as ffxsmod.f:26-54 does into ff_gff(81,41);
* ``data.ion``: ionisation potentials and level energies / weights of every
  ion of elements 1-30, as ions_read_data reads them (ionsmod.f:652-749);
* ``Atoms/data.atom.<el><ii>``: a seeded subset of the bound-bound lines of
  the ten elements of the physical-opacity workload (C, O, Ne, Mg, Si, S, Ca,
  Fe, Co, Ni), stages I-IV, with centres inside 1000-32000 A, packed into bb_xs records as
  read_bbxs_data.f:55-73 does (real*4 arithmetic) and sorted by wl0.

    python tests/golden/make_atomic_data.py [path/to/reference/Data]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DEFAULT_DATA = "/root/reference/Data"
OUT = os.path.join(HERE, "atomic_data.npz")
NLINE_SUBSET = 16_000
WL_RANGE_ANG = (1000.0, 32000.0)  # the group range of the workloads
SYMBOL = {6: "c", 8: "o", 10: "ne", 12: "mg", 14: "si", 16: "s", 20: "ca", 26: "fe", 27: "co", 28: "ni"}


def read_ions(path):
    """data.ion records: (icod, ionisation potential [cm^-1], level chi [cm^-1], level g)."""
    with open(path) as f:
        rows = f.read().split("\n")
    icod, ip, nlev, chi, g = [], [], [], [], []
    i = 0
    while i < len(rows):
        if not rows[i].strip():
            i += 1
            continue
        code = int(rows[i].split()[0])
        head = rows[i + 1]
        k = head.index("(Ky): ")
        n = int(rows[i + 3].split()[0])
        lev = rows[i + 4:i + 4 + n]
        icod.append(code)
        ip.append(float(head[k + 6:].split()[0]))
        nlev.append(n)
        for ln in lev:  # format (f11.3,1x,a12,i5,i5,l6): chi, label, ilevel, g, meta
            chi.append(float(ln[0:11]))
            g.append(int(ln[29:34]))
        i += 4 + n
    return (np.array(icod, np.int32), np.array(ip), np.array(nlev, np.int32), np.array(chi),
            np.array(g, np.int32))


def read_atom(path):
    """One data.atom file (bbxsmod.f:42-122): levels (chi real*4, id, g), lines (lev1, lev2, log gf real*4)."""
    with open(path) as f:
        rows = f.read().split("\n")
    nlevel, nline = (int(v) for v in rows[3].split()[:2])
    lev = rows[4:4 + nlevel]
    lin = rows[4 + nlevel:4 + nlevel + nline]
    chi = np.array([float(r[0:11]) for r in lev], np.float32)
    lid = np.array([int(r[24:29]) for r in lev], np.int64)
    g = np.array([int(r[29:34]) for r in lev], np.int32)
    l1 = np.array([int(r[0:5]) for r in lin], np.int64)
    l2 = np.array([int(r[5:10]) for r in lin], np.int64)
    f = np.array([float(r[10:17]) for r in lin], np.float32)
    rev = np.zeros(lid.max() + 1, np.int64)
    rev[lid] = np.arange(nlevel)
    return chi, g, rev[l1], rev[l2], f


def pack_lines(data_dir, nline, seed=5):
    """bb_xs records of the ten elements, stages I-IV (read_bbxs_data.f:55-73), seeded subset
    of the lines inside WL_RANGE_ANG."""
    from superlite_b200.workloads import BBXS_DTYPE, PC_PI, PC_E, PC_ME, PC_C
    fconst = np.float32(PC_PI * PC_E ** 2 / (PC_ME * PC_C))
    recs = []
    for iz, sym in SYMBOL.items():
        for ii in range(1, 5):
            p = os.path.join(data_dir, "Atoms", f"data.atom.{sym}{ii}")
            if not os.path.exists(p):
                continue
            chi, g, llw, lhg, f = read_atom(p)
            wl0 = np.float32(1e8) / (np.abs(chi[lhg]) - np.abs(chi[llw]))
            flip = wl0 < 0
            llw, lhg = np.where(flip, lhg, llw), np.where(flip, llw, lhg)
            wl0 = np.abs(wl0)
            r = np.zeros(len(f), BBXS_DTYPE)
            r["wl0"] = wl0
            r["gxs"] = fconst * g[llw].astype(np.float32) * np.float32(10.0) ** f
            r["chilw"] = np.abs(chi[llw])
            r["iz"], r["ii"] = iz, ii
            recs.append(r)
    allr = np.concatenate(recs)
    allr = allr[np.isfinite(allr["wl0"]) & (allr["wl0"] >= WL_RANGE_ANG[0]) & (allr["wl0"] <= WL_RANGE_ANG[1])]
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(len(allr), size=min(nline, len(allr)), replace=False))
    sub = allr[pick]
    return sub[np.argsort(sub["wl0"], kind="stable")], len(allr)


def main(data_dir):
    from superlite_b200 import workloads as W
    ph1, ph2 = W.load_verner(os.path.join(data_dir, "data.bf_verner"))
    gff = W.load_sutherland(os.path.join(data_dir, "data.ff_sutherland"))
    icod, ip, nlev, chi, g = read_ions(os.path.join(data_dir, "data.ion"))
    lines, nall = pack_lines(data_dir, NLINE_SUBSET)
    np.savez_compressed(OUT, bf_ph1=ph1, bf_ph2=ph2, ff_gff=gff, ion_icod=icod, ion_ip_cm=ip, ion_nlev=nlev,
                        lev_chi_cm=chi, lev_g=g.astype(np.int16), lines=lines, lines_total=np.int64(nall))
    print(f"wrote {OUT}: {len(icod)} ions, {len(chi)} levels, {len(lines)} of {nall} lines")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_DATA)
