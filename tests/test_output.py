"""The reference's flux and energy output files (OUTPUT/output_flux.f,
output_grid.f) written from the library's results read back the way
SuperLite's Tools do (numpy.loadtxt; edges from line 2 of output.flx_grid)."""
import numpy as np

from superlite_b200.output import EnergyOutput, FluxOutput, model_flux_writers


def test_flux_files_round_trip(tmp_path):
    wl = np.geomspace(1e-5, 3.2e-4, 101)
    rng = np.random.default_rng(3)
    w = FluxOutput(str(tmp_path), wl)
    steps = []
    for k in range(3):
        lum = rng.uniform(1e38, 1e41, 100)
        lum[5] = 0.0
        lum[6] = 1e-120   # would need a three-digit exponent: written as 0
        lum[7] = -3.0     # not above 1e-99: written as 0, as merge(..., x>1d-99) does
        dev = lum ** 2 / 10
        num = rng.integers(0, 5000, 100)
        w.write(lum, dev, num)
        steps.append((lum, dev, num))
    L = np.loadtxt(tmp_path / "output.flx_luminos")
    N = np.loadtxt(tmp_path / "output.flx_lumnum", dtype=np.int64)
    D = np.loadtxt(tmp_path / "output.flx_lumdev")
    assert L.shape == (3, 100) and N.shape == (3, 100) and D.shape == (3, 100)
    for k, (lum, dev, num) in enumerate(steps):
        ref = np.where(lum > 1e-99, lum, 0.0)
        np.testing.assert_allclose(L[k], ref, rtol=5e-5)
        np.testing.assert_array_equal(N[k], num)
        np.testing.assert_allclose(D[k], np.where(dev > 1e-99, dev, 0.0), rtol=5e-5)
    with open(tmp_path / "output.flx_grid") as f:
        head = f.readline()
        edges = np.array([float(v) for v in f.readline().split()])
    assert head.split()[1:] == ["100", "1", "1"]
    np.testing.assert_allclose(edges, wl, rtol=5e-5)
    # fixed-width 12-character fields, as '(1p,10000e12.4)' writes them
    line = open(tmp_path / "output.flx_luminos").readline().rstrip("\n")
    assert len(line) == 12 * 100


def test_energy_file_and_model_writers(tmp_path):
    e = EnergyOutput(str(tmp_path))
    e.write(1.0e50, -2.0e48, -1.0e50, 1.0e50)
    e.write(2.0e50, -3.0e48, -2.0e50, 2.0e50)
    T = np.loadtxt(tmp_path / "output.tot_energy")
    np.testing.assert_allclose(T, [[1.0e50, -2.0e48, -1.0e50, 1.0e50], [2.0e50, -3.0e48, -2.0e50, 2.0e50]],
                               rtol=5e-5)
    wl = np.geomspace(1e-5, 3.2e-4, 11)
    ws = model_flux_writers(str(tmp_path / "batch"), 3, wl)
    lum = np.arange(1, 31, dtype=float).reshape(3, 10) * 1e40
    for m, w in enumerate(ws):
        w.write(lum[m], lum[m], np.ones(10, dtype=int))
    for m in range(3):
        np.testing.assert_allclose(np.loadtxt(tmp_path / "batch" / f"model_{m:04d}" / "output.flx_luminos"), lum[m],
                                   rtol=5e-5)
