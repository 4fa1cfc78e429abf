"""The product library loads and exports every symbol include/*.h declares
(no device call is made)."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vpm_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "vpm_fmm2d_field" in names and "vpm_ctx_create" in names and len(names) >= 15


@pytest.mark.parametrize("name", declared_symbols())
def test_symbol_exported(name):
    import lsmps_vpm_v2_b200 as pkg
    lib = pkg.lib()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_python_binding_covers_header():
    from lsmps_vpm_v2_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_missing_library_fails_loudly(monkeypatch):
    from lsmps_vpm_v2_b200 import _lib
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "SO_PATH", os.path.join(ROOT, "no_such_lib.so"))
    with pytest.raises(RuntimeError):
        _lib.lib()


def test_params_default_are_reference_values():
    from lsmps_vpm_v2_b200 import default_params
    p = default_params()
    # global.cpp:303, 311-313; treeCell.cpp:5; global.cpp:779
    assert (p.p, p.max_src, p.max_par, p.exp_tree_pct, p.eps, p.leaf_cap_3d) == (10, 50, 75, 1.0, 1e-9, 30)
