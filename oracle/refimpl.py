"""TEST INFRASTRUCTURE ONLY -- the reference's own kernels compiled for the host cores.

Builds (here, where the reference tree is readable) and loads variants of
``oracle/ref/ref_driver.cpp``, which includes the reference's unmodified OpenCL C
sources through ``oracle/ref/clshim.hpp``.  Each discrete switch of the reference's
``-D`` settings (operator header, testcase header, USE_* flags, REAL) selects one
shared library ``oracle/_ref/ref_<key>.so``; mesh sizes, DX..DZ, XMIN..ZMAX, DT and the
dissipation parameters are set at run time (``ref_configure``).

Only tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg use this module.
On a machine without the reference tree only variants built beforehand are available.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
DRIVER = os.path.join(HERE, "ref", "ref_driver.cpp")
SHIM_DIR = os.path.join(HERE, "ref")
OWN_TESTCASES = os.path.join(HERE, "ref", "testcases")
REFERENCE_DIR = os.environ.get("IEQ_REFERENCE_DIR", "/root/reference")

REFERENCE_TESTCASES = ("rotation_2D", "rotation_3D", "hall_periodic", "hall_travelling_wave",
                       "confined_domain", "alfven_periodic_2D")
OWN_TESTCASE_NAMES = ("rotation_gaussian", "hall_circular_wave")


@dataclass(frozen=True)
class Variant:
    """The compile-time switches of one reference build (cf. generate_settings.m)."""
    real: str = "double"             # I_Tech('REAL')
    order: int = 4                   # I_RunOps('order')
    extended: bool = False           # I_RunOps('operator_form') == 'extended'
    testcase: str = "rotation_3D"    # I_RunOps('testcase')
    periodic: bool = False           # USE_PERIODIC
    hall: bool = False               # USE_HALL
    dissipation: str = "NONE"        # NONE | HIGH_ORDER | FIRST_ORDER | ADAPTIVE
    uibj: str = "PRODUCT"            # CENTRAL | SPLIT | PRODUCT
    source: str = "CENTRAL"          # ZERO | CENTRAL | SPLIT
    ujbi: str = "CENTRAL"            # CENTRAL | SPLIT | PRODUCT
    laplace: str = "WIDE_STENCIL_DIRICHLET"  # | NARROW_STENCIL_DIRICHLET | WIDE_STENCIL_LNS

    def header(self) -> str:
        return f"{self.order}{'th' if self.order > 2 else 'nd'}Order{'Extended' if self.extended else ''}.h"

    def defines(self) -> list[str]:
        d = [f"-DREAL={self.real}", f"-DIEQ_ORDER_HEADER={self.header()}",
             f"-DIEQ_TESTCASE_HEADER={self.testcase}.h",
             f"-DUSE_UIBJ_{self.uibj}=1", f"-DUSE_SOURCE_{self.source}=1",
             f"-DUSE_UJBI_{self.ujbi}=1", f"-DUSE_LAPLACE_{self.laplace}=1"]
        if self.periodic:
            d.append("-DUSE_PERIODIC=1")
        if self.hall:
            d.append("-DUSE_HALL=1")
        if self.dissipation != "NONE":
            d += ["-DUSE_ARTIFICIAL_DISSIPATION=1", f"-DUSE_{self.dissipation}_DISSIPATION=1"]
        return d

    def key(self) -> str:
        tag = (f"{'f32' if self.real == 'float' else 'f64'}_o{self.order}{'e' if self.extended else 'c'}_"
               f"{self.testcase}_{'per' if self.periodic else 'sat'}_{'hall' if self.hall else 'lin'}_"
               f"{self.dissipation.lower()}_{self.uibj[0]}{self.source[0]}{self.ujbi[0]}_"
               f"{self.laplace.split('_')[0][0]}{self.laplace.split('_')[-1][0:2].lower()}")
        return tag


def _lib_path(v: Variant) -> str:
    return os.path.join(REF_OUT, f"ref_{v.key()}.so")


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_DIR, "kernel", "kernel_time_integrator.cl"))


def build(v: Variant, force: bool = False) -> str:
    """Compile the variant from the reference sources in place; returns the .so path."""
    out = _lib_path(v)
    if os.path.isfile(out) and not force:
        return out
    if not reference_available():
        raise RuntimeError(f"reference tree not found at {REFERENCE_DIR}; "
                           f"variant {v.key()} was not built beforehand")
    os.makedirs(REF_OUT, exist_ok=True)
    tmp = out + f".{os.getpid()}.tmp"
    cmd = ["g++", "-O2", "-std=gnu++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-w",
           f"-I{SHIM_DIR}", f"-I{REFERENCE_DIR}/include", f"-I{REFERENCE_DIR}/kernel",
           f"-I{OWN_TESTCASES}", *v.defines(), DRIVER, "-o", tmp]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    os.replace(tmp, out)
    return out


_LIBS: dict[str, ctypes.CDLL] = {}


def load(v: Variant) -> ctypes.CDLL:
    path = build(v)
    lib = _LIBS.get(path)
    if lib is None:
        lib = ctypes.CDLL(path)
        lib.ref_configure.argtypes = [ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_uint]
        lib.ref_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint),
                                ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int]
        lib.ref_run.restype = ctypes.c_int
        lib.ref_kernel_name.restype = ctypes.c_char_p
        _LIBS[path] = lib
    return lib


@dataclass
class Mesh:
    """I_Mesh plus the time step and the parameters that the reference takes as -D values."""
    nodes: tuple[int, int, int]
    xmin: tuple[float, float, float]
    xmax: tuple[float, float, float]
    periodic: bool
    dt: float = 0.0
    hod_factor: float = 1.0
    mp2min: float = 1.0
    mp2max: float = 10.0
    cmin: float = 1.0
    cmax: float = 10.0
    tc_omega: float = 1.0
    bnodes: int = 1
    d: tuple[float, float, float] = field(init=False)

    def __post_init__(self):
        # matlab/+induction_eq/initialize.m:12-21
        n = self.nodes
        if self.periodic:
            self.d = tuple(float(self.xmax[i] - self.xmin[i]) / float(n[i]) for i in range(3))
        else:
            self.d = tuple(float(self.xmax[i] - self.xmin[i]) / (float(n[i]) - 1) for i in range(3))

    @property
    def num_nodes(self) -> int:
        return self.nodes[0] * self.nodes[1] * self.nodes[2]


class RefRunner:
    """Runs reference kernels by name on numpy arrays, like MatCL's cl_run_kernel."""

    def __init__(self, v: Variant, mesh: Mesh, nthreads: int = 1):
        self.v = v
        self.mesh = mesh
        self.lib = load(v)
        self.nthreads = nthreads
        self.dtype = np.float32 if v.real == "float" else np.float64
        nodes = (ctypes.c_uint * 3)(*mesh.nodes)
        m = mesh
        p = (ctypes.c_double * 16)(m.d[0], m.d[1], m.d[2], m.xmin[0], m.xmax[0], m.xmin[1], m.xmax[1],
                                   m.xmin[2], m.xmax[2], m.dt, m.hod_factor, m.mp2min, m.mp2max,
                                   m.cmin, m.cmax, m.tc_omega)
        self.lib.ref_configure(nodes, p, m.bnodes)

    def vec(self, n=None) -> np.ndarray:
        return np.zeros((n or self.mesh.num_nodes, 4), dtype=self.dtype)

    def scalar(self, n=None, fill=0.0) -> np.ndarray:
        return np.full((n or self.mesh.num_nodes,), fill, dtype=self.dtype)

    def run(self, name: str, grange, *arrays: np.ndarray) -> None:
        for a in arrays:
            assert a.dtype == self.dtype and a.flags.c_contiguous, name
        g = (ctypes.c_uint * 3)(*[int(x) for x in grange])
        ptrs = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        rc = self.lib.ref_run(name.encode(), g, ptrs, len(arrays), self.nthreads)
        if rc != 0:
            raise RuntimeError(f"ref_run({name}) failed with {rc}")

    def run_list(self, names, grange, *arrays: np.ndarray) -> None:
        for n in names:
            self.run(n, grange, *arrays)


def variant_digest(v: Variant) -> str:
    return hashlib.sha1(v.key().encode()).hexdigest()[:10]
