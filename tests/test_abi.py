"""The C ABI library loads and exports every entry point include/*.h declares.

No compute calls: this runs on machines without a GPU.
"""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(adi_[A-Za-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"adi_create", "adi_step", "adi_time_step", "adi_set_mask", "adi_build_segments"} <= names


def test_library_exports_every_declared_symbol(adi_lib):
    lib = ctypes.CDLL(adi_lib.library_path())
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(adi_lib):
    from adi_b200 import _abi
    assert declared_functions() <= set(_abi.EXPORTED) | {"adi_last_error_string"}


def test_library_is_sm100a_build(adi_lib):
    lib = adi_lib._abi.load()
    assert b"sm_100a" in lib.adi_version()


def test_fluid_params_match_reference_formulas(adi_lib):
    p = adi_lib.fluid_params_normalized(200.0, 0.72, 1.4)
    assert (p.v_T, p.v_vis, p.t_vis) == (1.0, 1.0 / 200.0, 1.0 / (200.0 * 0.72))
    assert p.t_phi == (1.4 - 1.0) / (1.4 * 200.0)
    q = adi_lib.fluid_params_dimensional(0.05, 1000.0, 461.495, 0.6, 4200.0)
    assert (q.v_T, q.v_vis, q.t_vis, q.t_phi) == (461.495, 0.05 / 1000.0, 0.6 / (1000.0 * 4200.0), 0.05 / (1000.0 * 4200.0))


def test_entry_points_reject_a_null_handle(adi_lib):
    """Handle-taking entry points answer ADI_ERR_BAD_ARG for a NULL handle or batch
    before they touch the device (so this runs without a GPU)."""
    from adi_b200 import _abi
    lib = _abi.load()
    vp = ctypes.c_void_p
    four = (vp * 4)()
    d, i = ctypes.c_double(1e-3), ctypes.c_int(0)
    calls = [
        ("adi_step_io", (None, four, four, d, 1, 1, 0)),
        ("adi_io_wait", (None,)),
        ("adi_phase_begin", (None, 1)),
        ("adi_phase_sweep", (None, 0, d, 1)),
        ("adi_phase_end", (None,)),
        ("adi_set_fault_injection", (None, 0)),
        ("adi_set_adjoint_chunk", (None, -4)),
        ("adi_batch_set_schedule", (None, 1, 2)),
        ("adi_batch_get_schedule", (None, ctypes.byref(i), ctypes.byref(i))),
        ("adi_batch_time_step", (None, d, 1, 1, 1, ctypes.byref(ctypes.c_float()))),
    ]
    for name, args in calls:
        assert getattr(lib, name)(*args) == _abi.ADI_ERR_BAD_ARG, name
