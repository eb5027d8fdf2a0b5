"""The C-ABI library loads and exports every entry point include/*.h declares (CPU only)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for h in sorted(os.listdir(INCLUDE)):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(pgpu_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib_path():
    from proteusgpu_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from proteusgpu_b200 import build
        build.build()
    return _lib.LIB_PATH


def test_header_declares_the_api():
    names = declared_functions()
    assert "pgpu_create" in names and "pgpu_sim_step" in names and "pgpu_periodic_mesh" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib_path):
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    assert set(declared_functions()) <= exported


def test_python_binding_covers_the_header(lib_path):
    from proteusgpu_b200 import _lib
    assert sorted(_lib.EXPORTED) == declared_functions()
    L = _lib.load()
    assert L.pgpu_abi_version() == 1


def test_default_params_are_the_references_defaults(lib_path):
    from proteusgpu_b200 import _lib
    L = _lib.load()
    p = _lib.Params()
    L.pgpu_default_params(ctypes.byref(p))
    # Config.sh:4,34 (dim_3D, _K_=190), allvars.cpp:13-14 (buff, _gamma_)
    assert (p.dim, p.k, p.boundary, p.flux_mode) == (3, 190, 0, 0)
    assert p.buff == 0.04 and p.gamma == 5.0 / 3.0


def test_create_rejects_bad_parameters_without_a_device(lib_path):
    from proteusgpu_b200 import _lib
    L = _lib.load()
    p = _lib.Params()
    L.pgpu_default_params(ctypes.byref(p))
    h = ctypes.c_void_p()
    for field, bad in (("dim", 4), ("k", 0), ("k", 257), ("buff", -1.0), ("gamma", 1.0), ("boundary", 7)):
        q = _lib.Params.from_buffer_copy(p)
        setattr(q, field, bad)
        assert L.pgpu_create(ctypes.byref(q), ctypes.byref(h)) == -1, field
    assert L.pgpu_create(None, ctypes.byref(h)) == -1
