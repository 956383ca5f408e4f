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
# the reference checkout: IEQ_REFERENCE_DIR, else a directory named "reference" beside this
# repository's root
REFERENCE_DIR = os.environ.get("IEQ_REFERENCE_DIR",
                               os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))

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


# Two builds of every variant:
#   strict (parity): -O2 -ffp-contract=off, the reference's evaluation order without fused
#     multiply-adds -- the oracle the tests compare against;
#   fast (timing): -O3 -ffp-contract=fast with the widest x86-64 level the host supports
#     (x86-64-v4: AVX-512; x86-64-v3: AVX2 + FMA), the build the CPU baseline and the
#     reference arm of bench.py time.  -march=native cannot be used: the library is built on
#     one machine and timed on another, whose CPU model may differ; both levels are built
#     and the one the running host supports is loaded.
FAST_LEVELS = ("x86-64-v4", "x86-64-v3")


def host_level() -> str:
    """x86-64-v4 if the running CPU has the AVX-512 subsets that level needs, else v3."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln.split(":", 1)[1].split() for ln in f if ln.startswith("flags")), [])
    except OSError:
        flags = []
    need = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")
    return "x86-64-v4" if all(x in flags for x in need) else "x86-64-v3"


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _lib_path(v: Variant, level: str | None = None) -> str:
    if level is None:
        return os.path.join(REF_OUT, f"ref_{v.key()}.so")
    return os.path.join(REF_OUT, f"ref_{v.key()}_fast_{level.replace('-', '')}.so")


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_DIR, "kernel", "kernel_time_integrator.cl"))


def build(v: Variant, force: bool = False, level: str | None = None) -> str:
    """Compile the variant from the reference sources in place; returns the .so path.
    level None: the strict parity build; an x86-64 level: the fast timing build."""
    out = _lib_path(v, level)
    if os.path.isfile(out) and not force:
        return out
    if not reference_available():
        raise RuntimeError(f"reference tree not found at {REFERENCE_DIR}; "
                           f"variant {v.key()} was not built beforehand")
    os.makedirs(REF_OUT, exist_ok=True)
    tmp = out + f".{os.getpid()}.tmp"
    opt = ["-O2", "-ffp-contract=off"] if level is None else ["-O3", f"-march={level}", "-ffp-contract=fast"]
    cmd = ["g++", *opt, "-std=gnu++17", "-fopenmp", "-fPIC", "-shared", "-w",
           f"-I{SHIM_DIR}", f"-I{REFERENCE_DIR}/include", f"-I{REFERENCE_DIR}/kernel",
           f"-I{OWN_TESTCASES}", *v.defines(), DRIVER, "-o", tmp]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    os.replace(tmp, out)
    return out


_LIBS: dict[str, ctypes.CDLL] = {}


def build_fast(v: Variant) -> list[str]:
    """Both fast timing builds of the variant."""
    return [build(v, level=lv) for lv in FAST_LEVELS]


def load(v: Variant, fast: bool = False) -> ctypes.CDLL:
    path = build(v, level=host_level() if fast else None)
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

    def __init__(self, v: Variant, mesh: Mesh, nthreads: int = 1, fast: bool = False):
        self.v = v
        self.mesh = mesh
        self.fast = fast
        self.lib = load(v, fast)
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
