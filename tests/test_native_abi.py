"""The C-ABI library loads (no GPU needed) and exports every entry point the
header declares, with the Python binding covering exactly that set."""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT

import dem._native as N

HEADER = ROOT / "include" / "dem_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^DEM_API\s+[\w\s\*]*?\b(dem_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "dem_direct_forces" in names and "dem_hash_detect" in names and "dem_merge" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(N.LIB_PATH))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_matches_header():
    assert set(N.SIGNATURES) == set(declared())
    N.lib()  # binds every signature
    assert N.version().startswith("dem_b200")


def test_build_targets_sm100a_only():
    # every object of the library is compiled with exactly this architecture flag
    import build_native

    assert build_native.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_runtime_loads_sm100_code():
    # the runtime's own answer for a kernel of the library: the code it loads is sm_100
    assert N.kernel_binary_version(0) == 100
