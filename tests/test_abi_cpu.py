"""CPU tests of the C ABI: the library loads, exports every declared entry point, and
rejects bad settings before touching a GPU (no compute calls here)."""
from __future__ import annotations

import ctypes

import pytest

from inductioneq_b200 import lib as L
from inductioneq_b200.induction_eq import Maps, generate_settings


def test_library_exports_every_declared_function():
    so = L.load()
    names = L.declared_functions()
    assert len(names) > 95 + 20
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_every_reference_kernel_has_a_typed_entry_point():
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "g", os.path.join(L.PKG, "csrc", "gen_kernel_abi.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    assert len(g.KERNELS) == 95
    so = L.load()
    for name, _, cite, _ in g.KERNELS:
        assert hasattr(so, "ieq_" + name), name
        assert cite.startswith("kernel/")


def _create(settings, paths):
    so = L.load()
    h = ctypes.c_void_p()
    arr = (ctypes.c_char_p * len(paths))(*[p.encode() for p in paths])
    st = so.ieq_create(ctypes.byref(h), settings.encode(), arr, len(paths), 0)
    return st, so.ieq_last_error(None).decode()


BASE = " -DNODES_X=16 -DNODES_Y=16 -DNODES_Z=16 -DXMIN=0 -DXMAX=1 -DYMIN=0 -DYMAX=1 -DZMIN=0 -DZMAX=1"


@pytest.mark.parametrize("settings,paths,status,msg", [
    (BASE, ["../include/rotation_3D.h"], 1, "operator header"),
    (BASE, ["../include/4thOrder.h"], 1, "testcase"),
    (" -DNODES_X=16", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "lack"),
    (BASE + " -DUSE_UIBJ_ZERO=1", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "flux form"),
    (BASE + " -DUSE_LAPLACE_NARROW_STENCIL_DIRICHLET=1", ["../include/4thOrderExtended.h", "../include/rotation_3D.h"],
     1, "narrow-stencil"),
    (BASE + " -DIEQ_INTEGRATOR=RK4", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "integrator"),
    (BASE.replace("=16", "=10"), ["../include/6thOrder.h", "../include/rotation_3D.h"], 2, "2*NUM_BOUNDS"),
    (BASE.replace("=16", "=10") + " -DUSE_PERIODIC=1", ["../include/6thOrder.h", "../include/rotation_3D.h"], 2,
     "STENCIL_WIDTH"),
    (BASE + " -DIEQ_COL_BLOCK=32x4x2", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "X * Y * Z = 128"),
    (BASE + " -DIEQ_CURL_BLOCK=32x4", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "XxYxZ"),
    (BASE + " -DIEQ_COL_PAIRS=3", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_COL_PAIRS"),
    (BASE + " -DIEQ_XBAND=3", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_XBAND"),
    (BASE + " -DIEQ_PDL=2", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_PDL"),
    (BASE + " -DIEQ_STAGE_KERNEL=FAST", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "ZMARCH"),
    (BASE + " -DIEQ_ZMARCH_TZ=-1", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_ZMARCH_TZ"),
    (BASE + " -DIEQ_HODP=2", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_HODP"),
    (BASE + " -DIEQ_CURL_Z=3", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_CURL_Z"),
    (BASE + " -DIEQ_CG_PASS_A=3", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1, "IEQ_CG_PASS_A"),
    (BASE + " -DIEQ_ADJOINT_PROGRAM=2", ["../include/4thOrder.h", "../include/rotation_3D.h"], 1,
     "IEQ_ADJOINT_PROGRAM"),
])
def test_bad_settings_are_rejected_on_the_host(settings, paths, status, msg):
    st, err = _create(settings, paths)
    assert st == status, (st, err)
    assert msg in err


def test_generate_settings_matches_reference_format():
    m = {"NODES_X": 40, "DX": 2.0 / 39.0, "form_uibj": "USE_UIBJ_PRODUCT", "REAL": "double",
         "optimizations": " -cl-mad-enable"}
    s = generate_settings(m, ["form_uibj", "NODES_X", "DX", "REAL", "optimizations"])
    assert s == " -DUSE_UIBJ_PRODUCT=1 -DNODES_X=40 -DDX=5.1282051282051280e-02 -DREAL=double -cl-mad-enable"


def test_maps_kernel_path_list_mirrors_setup():
    m = Maps()
    m.I_RunOps["order"] = 6
    m.I_RunOps["operator_form"] = "extended"
    m.I_IEq["dissipation"] = "USE_ARTIFICIAL_DISSIPATION"
    p = m.kernel_path_list()
    assert p[0] == "../include/6thOrderExtended.h"
    assert "../kernel/artificial_dissipation.cl" in p
    assert p[-1] == "../kernel/kernel_time_integrator.cl"


def test_kernel_selection_settings_are_emitted_and_accepted():
    # the I_Tech keys of the kernel choices become settings keys the library parses (on a
    # machine without a GPU ieq_create then stops at the device, not at the settings)
    m = Maps()
    m.I_Mesh.update({"NODES_X": 16, "NODES_Y": 16, "NODES_Z": 16, "XMIN": -1.0, "XMAX": 1.0, "YMIN": -1.0,
                     "YMAX": 1.0, "ZMIN": -1.0, "ZMAX": 1.0})
    m.I_TI["DT"] = 0.01
    m.I_RunOps["testcase"] = "rotation_3D"
    m.I_Tech.update({"stage_kernel": "ZMARCH", "col_block": (16, 4, 2), "curl_block": (8, 8, 2), "col_pairs": 4,
                     "xband": 2, "pdl": 0, "zmarch_tz": 24, "adjoint_program": 1, "hodp": 0})
    s = m.settings()
    for key in (" -DIEQ_STAGE_KERNEL=ZMARCH", " -DIEQ_COL_BLOCK=16x4x2", " -DIEQ_CURL_BLOCK=8x8x2",
                " -DIEQ_COL_PAIRS=4", " -DIEQ_XBAND=2", " -DIEQ_PDL=0", " -DIEQ_ZMARCH_TZ=24",
                " -DIEQ_ADJOINT_PROGRAM=1", " -DIEQ_HODP=0"):
        assert key in s, key
    st, err = _create(s, m.kernel_path_list())
    assert st not in (1, 2), (st, err)    # neither a settings nor a shape error
