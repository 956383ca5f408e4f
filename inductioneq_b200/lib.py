"""ctypes binding of the C ABI in include/inductioneq.h.

``load()`` returns the in-tree shared library ``_lib/libinductioneq_b200.so`` and raises if
it is missing -- there is no fallback implementation.  ``Context`` wraps one ``ieq_ctx``:
device buffers, the MatCL-form kernel-list call (``run``), the host-array form that copies
in and out like the MatCL mex (``run_host``), and the fused paths.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libinductioneq_b200.so")
HEADERS = [os.path.join(os.path.dirname(PKG), "include", h)
           for h in ("inductioneq.h", "inductioneq_kernels.h")]

STATUS = {0: "IEQ_OK", 1: "IEQ_ERR_SETTINGS", 2: "IEQ_ERR_SHAPE", 3: "IEQ_ERR_CUDA", 4: "IEQ_ERR_NAN",
          5: "IEQ_ERR_NOT_CONVERGED", 6: "IEQ_ERR_TIMEOUT", 7: "IEQ_ERR_UNKNOWN_KERNEL",
          8: "IEQ_ERR_ARG"}

_LIB = None


class KernelRecord(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 40), ("ms", ctypes.c_double)]


class IeqError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


def declared_functions() -> list[str]:
    names = []
    for h in HEADERS:
        with open(h) as f:
            names += re.findall(r"\b(ieq_\w+)\s*\(", f.read())
    return sorted(set(n for n in names if n not in ("ieq_status", "ieq_ctx", "ieq_results")))


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.isfile(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m inductioneq_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.ieq_create.argtypes = [ctypes.POINTER(vp), ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                               ctypes.c_int]
    lib.ieq_destroy.argtypes = [vp]
    lib.ieq_last_error.argtypes = [vp]
    lib.ieq_last_error.restype = ctypes.c_char_p
    for f in ("ieq_num_nodes", "ieq_num_nodes_pad", "ieq_num_groups"):
        getattr(lib, f).argtypes = [vp]
        getattr(lib, f).restype = sz
    lib.ieq_real_size.argtypes = [vp]
    lib.ieq_stream.argtypes = [vp]
    lib.ieq_stream.restype = vp
    lib.ieq_alloc.argtypes = [vp, sz, ctypes.POINTER(vp)]
    lib.ieq_free.argtypes = [vp, vp]
    lib.ieq_upload.argtypes = [vp, vp, vp, sz]
    lib.ieq_download.argtypes = [vp, vp, vp, sz]
    lib.ieq_memset.argtypes = [vp, vp, ctypes.c_int, sz]
    lib.ieq_synchronize.argtypes = [vp]
    lib.ieq_run_kernels.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(vp), ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_double)]
    lib.ieq_run_kernels_host.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(vp),
                                         ctypes.POINTER(sz), ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.ieq_time_steps.argtypes = [vp] * 8 + [ctypes.c_int]
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ieq_time_steps_integrals.argtypes = [vp] * 8 + [ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp]
    lib.ieq_clean_div.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    for f in ("ieq_norm2_value", "ieq_norm2_S_value"):
        getattr(lib, f).argtypes = [vp, vp, ctypes.POINTER(ctypes.c_double)]
    for f in ("ieq_norm2_diff_value", "ieq_dot_value"):
        getattr(lib, f).argtypes = [vp, vp, vp, ctypes.POINTER(ctypes.c_double)]
    lib.ieq_dot_range.argtypes = [vp, vp, vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    lib.ieq_compute_results.argtypes = [vp, vp, ctypes.c_double, vp, vp, ctypes.POINTER(ctypes.c_double * 4)]
    lib.ieq_check_finite.argtypes = [vp, vp]
    lib.ieq_test_brick_wait.argtypes = [vp, ctypes.c_int]
    lib.ieq_step_kernels.argtypes = [vp, ctypes.c_char_p, sz, ctypes.POINTER(ctypes.c_int)]
    lib.ieq_stages_begin.argtypes = [vp] * 6 + [ctypes.POINTER(ctypes.c_int)]
    lib.ieq_stages_run.argtypes = [vp, vp, vp, ctypes.c_int]
    lib.ieq_stages_field.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_longlong)]
    lib.ieq_stages_end.argtypes = [vp] * 7
    lib.ieq_profile_step.argtypes = [vp] * 8 + [ctypes.c_int, ctypes.c_int, ctypes.POINTER(KernelRecord),
                                                ctypes.POINTER(ctypes.c_int)]
    lib.ieq_operator_jvp.argtypes = [vp] * 6
    lib.ieq_operator_vjp.argtypes = [vp] * 6
    lib.ieq_ssprk33_step_vjp.argtypes = [vp, vp, vp, vp, ctypes.c_double, vp, vp, vp]
    lib.ieq_adjoint_steps.argtypes = [vp] * 5 + [ctypes.c_int, ctypes.c_int]
    lib.ieq_status_string.argtypes = [ctypes.c_int]
    lib.ieq_status_string.restype = ctypes.c_char_p
    lib.ieq_fp64_fma_rate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    _LIB = lib
    return lib


def _ptr(x) -> int:
    if isinstance(x, DeviceBuffer):
        return x.ptr
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if x is None:
        return 0
    return int(x)


class DeviceBuffer:
    """Device memory owned by a Context (freed with it)."""

    def __init__(self, ctx: "Context", nbytes: int):
        self.ctx = ctx
        self.nbytes = nbytes
        p = ctypes.c_void_p()
        ctx._check(ctx.lib.ieq_alloc(ctx.h, nbytes, ctypes.byref(p)))
        self.ptr = p.value

    def upload(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes, (a.nbytes, self.nbytes)
        self.ctx._check(self.ctx.lib.ieq_upload(self.ctx.h, self.ptr, a.ctypes.data, a.nbytes))

    def download(self, shape, dtype) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        self.ctx._check(self.ctx.lib.ieq_download(self.ctx.h, out.ctypes.data, self.ptr, out.nbytes))
        return out


class Context:
    """One InductionEq context (the compiled settings of cl_run_kernel(dev, paths, settings))."""

    def __init__(self, settings: str, kernel_paths, device: int = 0):
        self.lib = load()
        h = ctypes.c_void_p()
        paths = [p.encode() for p in kernel_paths]
        arr = (ctypes.c_char_p * len(paths))(*paths)
        st = self.lib.ieq_create(ctypes.byref(h), settings.encode(), arr, len(paths), device)
        if st != 0:
            raise IeqError(st, self.lib.ieq_last_error(None).decode())
        self.h = h.value
        self.n = self.lib.ieq_num_nodes(self.h)
        self.n_pad = self.lib.ieq_num_nodes_pad(self.h)
        self.n_groups = self.lib.ieq_num_groups(self.h)
        self.real = np.float32 if self.lib.ieq_real_size(self.h) == 4 else np.float64

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ieq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            raise IeqError(st, self.lib.ieq_last_error(self.h).decode())

    # ---------------------------------------------------------------- memory
    def alloc(self, nbytes: int) -> DeviceBuffer:
        return DeviceBuffer(self, nbytes)

    def vec(self, host: np.ndarray | None = None) -> DeviceBuffer:
        b = DeviceBuffer(self, self.n_pad * 4 * np.dtype(self.real).itemsize)
        if host is not None:
            b.upload(np.ascontiguousarray(host, dtype=self.real))
        return b

    def scalar(self, host: np.ndarray | None = None, n: int | None = None) -> DeviceBuffer:
        b = DeviceBuffer(self, (n or self.n_pad) * np.dtype(self.real).itemsize)
        if host is not None:
            b.upload(np.ascontiguousarray(host, dtype=self.real))
        return b

    def get_vec(self, b: DeviceBuffer) -> np.ndarray:
        return b.download((self.n_pad, 4), self.real)

    def get_scalar(self, b: DeviceBuffer, n: int | None = None) -> np.ndarray:
        return b.download((n or self.n_pad,), self.real)

    def synchronize(self) -> None:
        self._check(self.lib.ieq_synchronize(self.h))

    # ---------------------------------------------------------------- kernel lists
    def run(self, names, grange, *args, timed: bool = False) -> float | None:
        """cl_run_kernel(dev, names, g_range, l_range, args..., 0) on device buffers."""
        if isinstance(names, str):
            names = [names]
        nm = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        g = (ctypes.c_uint32 * 3)(*[int(x) for x in grange])
        av = (ctypes.c_void_p * len(args))(*[_ptr(a) for a in args])
        el = ctypes.c_double(0.0)
        self._check(self.lib.ieq_run_kernels(self.h, nm, len(names), g, av, len(args),
                                             ctypes.byref(el) if timed else None))
        return el.value if timed else None

    def run_host(self, names, grange, *arrays: np.ndarray) -> float:
        """The same on host arrays, copied in and back in place (the MatCL mex behaviour)."""
        if isinstance(names, str):
            names = [names]
        for a in arrays:
            assert a.flags.c_contiguous
        nm = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        g = (ctypes.c_uint32 * 3)(*[int(x) for x in grange])
        av = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        sz = (ctypes.c_size_t * len(arrays))(*[a.nbytes for a in arrays])
        el = ctypes.c_double(0.0)
        self._check(self.lib.ieq_run_kernels_host(self.h, nm, len(names), g, av, sz, len(arrays),
                                                  ctypes.byref(el)))
        return el.value

    def step_kernels(self) -> list[str]:
        """The reference kernel list of one time step of the configured integrator."""
        n = ctypes.c_int(0)
        self._check(self.lib.ieq_step_kernels(self.h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(64 * max(n.value, 1))
        self._check(self.lib.ieq_step_kernels(self.h, buf, len(buf), ctypes.byref(n)))
        return [k for k in buf.value.decode().split("\n") if k]

    # ---------------------------------------------------------------- stage by stage
    def stages_begin(self, b, b2, b3, curlB_rho, u) -> int:
        """Start stage-by-stage fused stepping (ieq_stages_begin); the stages of one step."""
        n = ctypes.c_int(0)
        self._check(self.lib.ieq_stages_begin(self.h, _ptr(b), _ptr(b2), _ptr(b3), _ptr(curlB_rho), _ptr(u),
                                              ctypes.byref(n)))
        return n.value

    def stages_run(self, rho, time, stage: int) -> None:
        self._check(self.lib.ieq_stages_run(self.h, _ptr(rho), _ptr(time), int(stage)))

    def stages_field(self, field: int) -> tuple[int, int]:
        """(device address of the x plane, component stride in elements) of state field
        `field` (0 b1, 1 b2, 2 b3) after the last stage run."""
        p, st = ctypes.c_void_p(), ctypes.c_longlong()
        self._check(self.lib.ieq_stages_field(self.h, int(field), ctypes.byref(p), ctypes.byref(st)))
        return p.value or 0, st.value

    def stages_end(self, b, b2, b3, curlB_rho, u, rho) -> None:
        self._check(self.lib.ieq_stages_end(self.h, _ptr(b), _ptr(b2), _ptr(b3), _ptr(curlB_rho), _ptr(u),
                                            _ptr(rho)))

    def kernel(self, name: str, *args) -> None:
        """The typed entry point ieq_<name> (reference NDRange)."""
        f = getattr(self.lib, "ieq_" + name)
        self._check(f(ctypes.c_void_p(self.h), *[ctypes.c_void_p(_ptr(a)) for a in args]))

    # ---------------------------------------------------------------- fused paths
    def time_steps(self, b, b2, b3, curlB_rho, u, rho, time, num_steps: int) -> None:
        self._check(self.lib.ieq_time_steps(self.h, _ptr(b), _ptr(b2), _ptr(b3), _ptr(curlB_rho), _ptr(u),
                                            _ptr(rho), _ptr(time), int(num_steps)))

    def time_steps_integrals(self, b, b2, b3, curlB_rho, u, rho, time, num_steps: int, clean_max_iterations: int = 0,
                             clean_threshold: float = 0.0) -> dict:
        """time_steps with the per-step series of save_integrals_over_time: energy, divergence
        norm and L2 error of b before every step (numpy arrays of num_steps entries); with
        clean_max_iterations > 0 B is cleaned after every step."""
        n = int(num_steps)
        e, d, l = (np.zeros(max(n, 1)) for _ in range(3))
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.ieq_time_steps_integrals(
            self.h, _ptr(b), _ptr(b2), _ptr(b3), _ptr(curlB_rho), _ptr(u), _ptr(rho), _ptr(time), n,
            int(clean_max_iterations), float(clean_threshold), e.ctypes.data_as(dp), d.ctypes.data_as(dp),
            l.ctypes.data_as(dp)))
        return {"energy": e[:n], "divergence_norm": d[:n], "l2_error": l[:n]}

    def clean_div(self, b, max_iterations: int, absolute_error_threshold: float, check: bool = True):
        it = ctypes.c_int(0)
        rr = ctypes.c_double(0)
        ini = ctypes.c_double(0)
        st = self.lib.ieq_clean_div(self.h, _ptr(b), int(max_iterations), float(absolute_error_threshold),
                                    ctypes.byref(it), ctypes.byref(rr), ctypes.byref(ini))
        if st not in (0, 5) or (check and st != 0):
            self._check(st)
        return {"iterations": it.value, "residual_norm2": rr.value, "divergence_norm_initial": ini.value,
                "converged": st == 0}

    def norm2(self, b) -> float:
        r = ctypes.c_double()
        self._check(self.lib.ieq_norm2_value(self.h, _ptr(b), ctypes.byref(r)))
        return r.value

    def norm2_diff(self, a, b) -> float:
        r = ctypes.c_double()
        self._check(self.lib.ieq_norm2_diff_value(self.h, _ptr(a), _ptr(b), ctypes.byref(r)))
        return r.value

    def norm2_S(self, s) -> float:
        r = ctypes.c_double()
        self._check(self.lib.ieq_norm2_S_value(self.h, _ptr(s), ctypes.byref(r)))
        return r.value

    def dot(self, a, b) -> float:
        r = ctypes.c_double()
        self._check(self.lib.ieq_dot_value(self.h, _ptr(a), _ptr(b), ctypes.byref(r)))
        return r.value

    def dot_range(self, a, b, first: int, count: int) -> float:
        """The dot product of elements [first, first + count) of two scalar fields."""
        r = ctypes.c_double()
        self._check(self.lib.ieq_dot_range(self.h, _ptr(a), _ptr(b), int(first), int(count), ctypes.byref(r)))
        return r.value

    def results(self, b, t: float, work_vec, work_scalar) -> dict:
        out = (ctypes.c_double * 4)()
        self._check(self.lib.ieq_compute_results(self.h, _ptr(b), float(t), _ptr(work_vec), _ptr(work_scalar),
                                                 ctypes.byref(out)))
        return {"abs_err": out[0], "rel_err": out[1], "divergence_norm": out[2], "energy": out[3]}

    def profile_step(self, b, b2, b3, curlB_rho, u, rho, time, repeats: int = 20) -> list[tuple[str, float]]:
        """Average device time (ms) of every launch of one step, each timed alone in a graph of
        `repeats` back-to-back launches; the fields hold no solution afterwards."""
        recs = (KernelRecord * 256)()
        n = ctypes.c_int(0)
        self._check(self.lib.ieq_profile_step(self.h, _ptr(b), _ptr(b2), _ptr(b3), _ptr(curlB_rho), _ptr(u),
                                              _ptr(rho), _ptr(time), int(repeats), 256, recs, ctypes.byref(n)))
        return [(recs[i].name.decode(), recs[i].ms) for i in range(min(n.value, 256))]

    # ---------------------------------------------------------------- discrete adjoint
    def operator_jvp(self, b, v, u, rho, out) -> None:
        self._check(self.lib.ieq_operator_jvp(self.h, _ptr(b), _ptr(v), _ptr(u), _ptr(rho), _ptr(out)))

    def operator_vjp(self, b, w, u, rho, out) -> None:
        self._check(self.lib.ieq_operator_vjp(self.h, _ptr(b), _ptr(w), _ptr(u), _ptr(rho), _ptr(out)))

    def ssprk33_step_vjp(self, s1, s2, s3, t0: float, lam, u, rho) -> None:
        self._check(self.lib.ieq_ssprk33_step_vjp(self.h, _ptr(s1), _ptr(s2), _ptr(s3), float(t0), _ptr(lam),
                                                  _ptr(u), _ptr(rho)))

    def adjoint_steps(self, b0, lam, u, rho, num_steps: int, checkpoint_every: int = 10) -> None:
        self._check(self.lib.ieq_adjoint_steps(self.h, _ptr(b0), _ptr(lam), _ptr(u), _ptr(rho), int(num_steps),
                                               int(checkpoint_every)))

    def memset(self, buf, value: int = 0) -> None:
        self._check(self.lib.ieq_memset(self.h, _ptr(buf), value, buf.nbytes))

    @property
    def stream(self) -> int:
        return self.lib.ieq_stream(self.h)

    def check_finite(self, b) -> None:
        self._check(self.lib.ieq_check_finite(self.h, _ptr(b)))

    def test_brick_wait(self, first_wait_gives_up: bool) -> None:
        """Failure-path test hook of the TMA brick kernels' waits (ieq_test_brick_wait)."""
        self._check(self.lib.ieq_test_brick_wait(self.h, 1 if first_wait_gives_up else 0))


def fp64_fma_rate(device: int = 0, iterations: int = 20000) -> float:
    """The device's FP64 rate in GFLOP/s, measured with an FMA loop (ieq_fp64_fma_rate)."""
    lib = load()
    g = ctypes.c_double(0.0)
    st = lib.ieq_fp64_fma_rate(int(device), int(iterations), ctypes.byref(g))
    if st != 0:
        raise IeqError(st, lib.ieq_status_string(st).decode())
    return g.value
