"""CPU tests of the boundary: the C-ABI library loads, exports every function
declared in include/cugridder.h (and the reference's eight names under
libcurafft.so), and the reference-style binding validates its arguments the
way the reference's ndpointer argtypes do.  No compute call is made."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cugridder.h")
REFERENCE_NAMES = ["ms2dirty_1", "ms2dirty_2", "dirty2ms_1", "dirty2ms_2", "ms2dirtyf_1",
                   "ms2dirtyf_2", "dirty2msf_1", "dirty2msf_2"]


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", src, flags=re.M)))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    for n in REFERENCE_NAMES:
        assert n in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from cugridder_b200 import _lib

    lib = _lib.load()
    for n in declared_functions():
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert set(declared_functions()) <= exported


def test_reference_file_name_alias():
    from cugridder_b200 import _lib

    alias = os.path.join(os.path.dirname(_lib.LIB_PATH), "libcurafft.so")
    lib = ctypes.CDLL(alias)
    for n in REFERENCE_NAMES:
        assert hasattr(lib, n)


def test_version_and_error_string():
    from cugridder_b200 import _lib

    lib = _lib.load()
    assert lib.cg_version() >= 100
    assert isinstance(lib.cg_last_error(), bytes)


def test_binding_rejects_wrong_dtypes_before_any_call():
    import cugridder_b200 as cg

    uvw = np.zeros((4, 3), dtype=np.float32)  # FP64 entry point wants float64
    ms = np.zeros(4, dtype=np.complex128)
    dirty = np.zeros((8, 8), dtype=np.complex128)
    with pytest.raises(TypeError):
        cg.ms2dirty_1(4, 8, 8, 1.0, 1e8, uvw, ms, dirty, 1e-5, 2.0, -1)
    with pytest.raises(TypeError):
        cg.ms2dirty_1(4, 8, 8, 1.0, 1e8, np.zeros((4, 3)), ms.astype(np.complex64), dirty, 1e-5,
                      2.0, -1)
    with pytest.raises(TypeError):
        cg.dirty2ms_1(4, 8, 8, 1.0, 1e8, np.zeros((4, 3)), ms, np.zeros((8, 8), complex)[:, ::2],
                      1e-5, 2.0, -1)


def test_curig_drop_in_names():
    import curig

    for n in ["ms2dirty", "dirty2ms", "vis2dirty", "dirty2vis"] + REFERENCE_NAMES:
        assert hasattr(curig, n), n


def test_no_oracle_in_product():
    """The product package never imports or loads the oracle."""
    pkg = os.path.join(ROOT, "cugridder_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in txt.lower() or f == "build.py", f
