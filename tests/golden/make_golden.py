"""Writes tests/golden/oracle_small.npz: outputs of the oracle (the C++
restatement of the reference's Fortran, test infrastructure) on small seeded
cases.  The reference itself cannot run in this image (no Fortran compiler)
and ships no golden vectors, so these fixtures pin the restatement against
unintended change; tests/test_golden.py recomputes them and requires exact
equality.  Regenerate only when the restatement is deliberately changed:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def compute():
    import pyoracle as po
    import cases
    from superlite_b200 import workloads as W
    po.build()
    out = {}
    # physical opacity and means: 8 shells x 24 groups x 400 lines
    oc = W.opacity_case(ncell=8, ng=24, nline=400, seed=31, t_days=9.0)
    r = po.physical_opacity(oc)
    out["opac_cap64"] = r["cap64"]
    out["opac_cap"] = r["cap"]
    out["opac_sig"] = r["sig"]
    out["opac_planck"] = po.planckmean(oc.groups.wlinv, oc.gas.temp, r["cap"])
    out["opac_ross"] = po.rossmean(oc.groups.wlinv, oc.gas.temp, r["sig"], r["cap"])
    # Saha EOS on the same shells (partition functions frozen at the first shell's T)
    ion = W.ion_table()
    q = po.partition(ion, float(oc.gas.temp[0]))
    nel, ocs, ginv, it = po.saha_eos(ion, q, oc.gas.temp, oc.gas.natom, oc.grid.vol, oc.gas.natomfr,
                                     np.ones(8), acc=1e-12, noc=oc.gas.oc.shape[1])
    out["eos_nelec"], out["eos_oc"], out["eos_ginv"] = nel, ocs, ginv
    # transport: 16 shells x 20 groups, 300 particles, shared Philox stream
    c = cases.transport_case(po, t_days=6.0, nx=16, ng=20, npart=300, seed=5)
    t = c["tables"]
    out["leak_opaclump"] = t["opaclump"]
    out["emitprob"] = t["emitprob"]
    tt = po.TransportTables(c["grid"], c["groups"], **t, params=c["params"])
    prt, isv = c["prt"].copy(), c["isv"].copy()
    rr = po.particle_advance(tt, prt, isv, rngmode=1, seed=7, nthreads=1, trace=True)
    out["trn_trace_hash"] = np.asarray(rr["trace_hash"])
    out["trn_counts"] = np.array([rr["npckt"], rr["nflux"], rr["nstepimc"], rr["nstepddmc"], rr["nstepmax"]],
                                 dtype=np.int64)
    out["trn_tally"] = np.asarray(rr["tally"])
    lum, dev, num = po.fluxtally(prt, isv, c["groups"].wl)
    out["trn_lum"], out["trn_lumnum"] = lum, num
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **compute())
    print("wrote", os.path.join(HERE, "oracle_small.npz"))
