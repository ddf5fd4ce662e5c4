"""Host-side helpers of bench.py (no GPU): the per-model luminosity z-scores
of the mixed form against the FP64 form, and the stratified model order of the
CPU-baseline sample."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_luminosity_zscores_known_values():
    import bench
    lum_a = np.array([[1.0, 1.0, 2.0, 2.0], [4.0, 0.0, 0.0, 0.0]])
    lum_b = np.array([[1.0, 1.0, 1.0, 1.0], [4.0, 0.0, 0.0, 0.0]])
    dev = np.array([[0.5, 0.5, 0.5, 0.5], [1.0, 0.0, 0.0, 0.0]])
    r = bench.luminosity_zscores({"lum": lum_a, "dev": dev}, {"lum": lum_b, "dev": dev}, np.array([1.0, 2.0]),
                                 nbin=2)
    # model 0: bins (1+1 vs 1+1) -> 0, (2+2 vs 1+1) -> 2 / sqrt(2); model 1: bin 0 -> 0, bin 1 has no variance
    assert r["comparisons"] == 3
    assert math.isclose(r["max_abs_z"], 2 / math.sqrt(2.0))
    assert r["frac_abs_z_gt_3"] == 0.0
    assert r["worst"][0]["model"] == 0 and r["worst"][0]["t_days"] == 1.0


def test_stratified_order_is_a_spread_permutation():
    import bench
    t = np.random.default_rng(1).uniform(1, 30, 128)
    order = bench.stratified_order(t)
    assert sorted(order) == list(range(128))
    first8 = np.sort(t[order[:8]])
    # the first eight models span the range: one from each eighth of the sorted times
    ranks = np.searchsorted(np.sort(t), first8)
    assert np.all(np.diff(ranks // 16) == 1) and ranks[0] < 16


def test_profile_commands_parse():
    """Every `python bench.py ...` command that a summary under profiles/ gives
    as the one that made its figures is accepted by bench.py's parser (the
    summaries stay reproducible from the committed files)."""
    import re
    import shlex
    import bench
    prof = os.path.join(ROOT, "profiles")
    cmds = []
    for name in sorted(os.listdir(prof)):
        if not name.endswith(".md"):
            continue
        text = open(os.path.join(prof, name)).read().replace("\\\n", " ")
        for m in re.finditer(r"python bench\.py([^\n#`]*)", text):
            args = m.group(1).split(">")[0].split("&&")[0]
            cmds.append((name, shlex.split(args)))
    assert cmds
    saved = sys.argv
    try:
        for name, args in cmds:
            sys.argv = ["bench.py"] + [a for a in args if not a.startswith("<")]
            bench.parse()  # exits (SystemExit) on an unknown flag
    finally:
        sys.argv = saved
