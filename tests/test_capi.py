"""CPU checks of the C ABI: the library builds for sm_100a, loads, and exports
every entry point declared in include/slg.h.  No kernel is launched here."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "slg.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(slg_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from superlite_b200 import build, capi
    build.build()
    return capi.load()


def test_header_declares_expected_entry_points():
    names = _declared()
    for must in ("slg_physical_opacity", "slg_opacity_means", "slg_leakage_opacity11",
                 "slg_emission_probability", "slg_particle_advance", "slg_fluxtally", "slg_sourcetally"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    from superlite_b200 import build
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (slg_[a-z0-9_]+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing


def test_binding_covers_header(lib):
    from superlite_b200 import capi
    assert sorted(capi.SIGNATURES) == _declared()


def test_no_device_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from superlite_b200 import HotPath, SlgError
    with pytest.raises(SlgError):
        HotPath(0)


def test_version_string(lib):
    assert b"sm_100a" in lib.slg_version()


def test_null_context_errors(lib):
    assert lib.slg_set_groups(None, 0, None) == -2
    assert lib.slg_sync(None) == -2
