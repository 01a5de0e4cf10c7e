"""The C-ABI library loads and exports every function include/gp_b200.h declares
(no device calls: runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT
import microsim_b200 as mb


def declared_functions():
    text = open(os.path.join(ROOT, "include", "gp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(gp_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_api():
    names = declared_functions()
    for n in ("gp_create", "gp_step", "gp_upload", "gp_download", "gp_get_stats", "gp_input_read",
              "gp_model_from_input", "gp_fill", "gp_write_vtk", "gp_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(mb.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_layout_matches_library():
    assert mb.lib().gp_model_sizeof() == ctypes.sizeof(mb.GpModel)


def test_driver_binary_present():
    assert os.access(mb.DRIVER_PATH, os.X_OK)
