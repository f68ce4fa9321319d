"""The C-ABI library loads and exports every entry point that include/heff.h declares (CPU only)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(heff_[A-Za-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return syms


@pytest.fixture(scope="module")
def libpath():
    import dmrg_b200
    from dmrg_b200 import build as b

    if not os.path.exists(dmrg_b200.LIB_PATH):
        b.build()
    return dmrg_b200.LIB_PATH


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("heff_matvec_d", "heff_matvec_z", "heff_op_create", "heff_op_multax", "heff_perform_op", "heff_expval_d"):
        assert s in syms


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"


def test_python_binding_signatures(libpath):
    import dmrg_b200

    L = dmrg_b200.lib()
    assert L.heff_version().decode().startswith("heff_b200")
    assert L.heff_last_error() is not None


def test_library_links_no_torch(libpath):
    """The product library is plain CUDA: no torch / python symbols in its dynamic dependencies."""
    import subprocess

    out = subprocess.run(["ldd", libpath], capture_output=True, text=True).stdout
    assert "torch" not in out and "python" not in out
