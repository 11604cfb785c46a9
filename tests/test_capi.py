"""The C ABI library loads and exports every entry point include/hif_b200.h declares.

CPU-only: no compute call is made without a GPU; hif_create must refuse cleanly.
"""
import ctypes
import os
import re
import subprocess

import pytest

import hifde3d_b200 as hb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(ROOT, "include", fn)) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\*?\s+\**(hif_[a-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("hif_create", "hif_factor", "hif_apply", "hif_setup_stencil", "hif_solve_pcg",
                 "hif_destroy", "hif_spmv"):
        assert must in names


def test_library_exports_every_declared_symbol():
    path = hb.library_path()
    assert os.path.exists(path), "build the library first (python -m hifde3d_b200.build)"
    L = ctypes.CDLL(path)
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hif_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported


def test_python_signatures_cover_header():
    assert set(declared_functions()) - {"hif_last_error"} <= set(hb._SIGNATURES)


def test_create_without_gpu_is_refused_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(hb.HIFError) as e:
        hb.HIFFactor(7, 4, 1e-6)
    assert e.value.code == hb.HIF_ERR_NODEVICE


def test_bad_arguments_are_rejected():
    L = hb.lib()
    h = ctypes.c_void_p()
    assert L.hif_create(0, 4, 1e-6, 0, ctypes.byref(h)) == hb.HIF_ERR_ARG
    assert L.hif_create(7, 4, -1.0, 0, ctypes.byref(h)) == hb.HIF_ERR_ARG
    assert L.hif_create(7, 4, 1e-6, 9, ctypes.byref(h)) == hb.HIF_ERR_ARG
    assert L.hif_factor(None) == hb.HIF_ERR_ARG
    assert L.hif_apply(None, None, 1, 1, 0) == hb.HIF_ERR_ARG
    assert L.hif_save_factor(None, b"/tmp/f.hif") == hb.HIF_ERR_ARG
    assert L.hif_load_factor(None, b"/tmp/f.hif") == hb.HIF_ERR_ARG
