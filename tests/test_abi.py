"""The C ABI library: it loads, it exports every entry point include/spo_b200.h declares, the
ctypes descriptor matches the header's struct, and invalid descriptors are refused before any
device is touched (CPU only; no compute call needs a GPU here)."""

import ctypes
import os
import re

import pytest

from conftest import ROOT, _ensure_built


def header_functions():
    text = open(os.path.join(ROOT, "include", "spo_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(spo_\w+)\s*\(", text, flags=re.M)))


def test_header_and_binding_agree():
    from spo_b200 import capi
    assert header_functions() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    _ensure_built()
    from spo_b200 import capi
    lib = capi.load_library()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert lib.spo_version().decode() == "0.1.0"


def test_descriptor_layout_matches_header():
    """Field names and order of struct spo_desc in the header equal the ctypes structure."""
    from spo_b200 import capi
    text = open(os.path.join(ROOT, "include", "spo_b200.h")).read()
    body = text[text.index("typedef struct spo_desc {"):text.index("} spo_desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl or decl.startswith("typedef"):
            decl = decl.split("{", 1)[-1].strip()
            if not decl:
                continue
        parts = decl.replace("*", " ").split()
        rest = " ".join(parts[1:]) if parts[0] != "const" else " ".join(parts[2:])
        names += [n.strip() for n in rest.split(",") if n.strip()]
    assert names == [f[0] for f in capi.SpoDesc._fields_]


def test_invalid_descriptor_is_refused_without_a_device():
    _ensure_built()
    from spo_b200 import capi
    lib = capi.load_library()
    d = capi.SpoDesc()  # all zero: n_rot = 0
    h = ctypes.c_void_p()
    st = lib.spo_create(ctypes.byref(d), ctypes.byref(h))
    assert st == capi.SPO_ERR_INVALID
    assert "positive" in lib.spo_last_error(None).decode()
    assert not h.value
    assert lib.spo_create(None, ctypes.byref(h)) == capi.SPO_ERR_INVALID


def test_null_handle_calls_are_refused():
    _ensure_built()
    from spo_b200 import capi
    lib = capi.load_library()
    assert lib.spo_propagate_analysis_step(None) == capi.SPO_ERR_INVALID
    assert lib.spo_destroy(None) == capi.SPO_OK


def mlp_header_functions():
    text = open(os.path.join(ROOT, "include", "spo_mlp.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(spo_mlp_\w+)\s*\(", text, flags=re.M)))


def test_mlp_header_binding_and_library_agree():
    """include/spo_mlp.h, the Python binding (spo_b200/mlp.py) and the library's symbols."""
    _ensure_built()
    from spo_b200 import capi, mlp
    assert mlp_header_functions() == sorted(mlp._EXPORTS)
    lib = capi.load_library()
    for name in mlp_header_functions():
        assert hasattr(lib, name), name


def test_mlp_invalid_shapes_are_refused_without_a_device():
    _ensure_built()
    from spo_b200 import capi, mlp
    lib = mlp._bind(capi.load_library())
    h = ctypes.c_void_p()
    assert lib.spo_mlp_create(65, 256, 4, 1, 0, ctypes.byref(h)) == capi.SPO_ERR_INVALID
    assert "n_in" in lib.spo_mlp_last_error(None).decode()
    assert lib.spo_mlp_create(8, 200, 4, 1, 0, ctypes.byref(h)) == capi.SPO_ERR_INVALID
    assert "width" in lib.spo_mlp_last_error(None).decode()
