"""The C ABI library loads and exports every symbol include/*.h declares;
without a GPU the compute entry points fail loudly (no CPU fallback)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for path in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(fh_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["fh_system_create", "fh_sweep", "fh_partial_inductance_matrix", "fh_lu_solve_c64", "fh_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from fasterhenry_b200 import _native as N
    lib = ctypes.CDLL(N.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_build_info(fh):
    from fasterhenry_b200 import _native as N
    assert N.load().fh_abi_version() == 1
    assert "sm_100a" in fh.build_info()


def test_no_device_means_no_fallback(fh):
    if fh.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(fh.NoDevice):
        fh.partial_inductance_matrix(np.zeros((1, 19)))
    with pytest.raises(fh.NoDevice):
        fh.lu_solve(np.eye(2), np.ones(2))
