"""ctypes binding of libmpsb200.so (the C ABI declared in include/mpsb200.h).

The library is loaded from the package directory.  There is no fallback: if
the shared object is missing or no sm_100 device is present, every entry point
raises, so the GPU path can never silently become a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmpsb200.so")

MPSB_CHI_LIMIT = 64
FP64 = 0
MIXED_TF32X3 = 1
TF32X3_ALL = 2
ST_NOCONV, ST_NONFINITE, ST_BADDIM, ST_TIMEOUT, ST_CHI_LIMIT = 1, 2, 4, 8, 16


def keep_limit(n: int, chi_max: int) -> int:
    """Largest bond an update of an n-site chain with this chi_max forms on the
    device: min(chi_max, MPSB_CHI_LIMIT, 2^(n//2)) (the kernels' keep_limit)."""
    schmidt = 1 << 7 if n >= 14 else (1 if n < 2 else 1 << (n // 2))
    return min(int(chi_max), MPSB_CHI_LIMIT, schmidt)
_ERRORS = {-1: "EINVAL", -2: "ELAUNCH", -3: "EWORKSPACE", -4: "ENODEV"}

# Symbols the header declares; tests check that every one is exported.
EXPORTS = (
    "mpsb_version", "mpsb_last_error", "mpsb_update2q_workspace_bytes", "mpsb_update2q_batch",
    "mpsb_apply1q_batch", "mpsb_statevector", "mpsb_amplitude", "mpsb_expect_workspace_bytes",
    "mpsb_expect_local", "mpsb_fp64_probe", "mpsb_update2q_batch_noalloc", "mpsb_overlap",
    "mpsb_update2q_tape_bytes", "mpsb_update2q_batch_taped", "mpsb_update2q_backward_workspace_bytes",
    "mpsb_update2q_backward_batch", "mpsb_apply1q_backward_batch", "mpsb_mpo_grad_workspace_bytes",
    "mpsb_mpo_energy_grad", "mpsb_sample_workspace_bytes", "mpsb_sample", "mpsb_reset_batch",
    "mpsb_canonicalize_workspace_bytes", "mpsb_canonicalize",
    "mpsb_update2q_flow_workspace_bytes", "mpsb_update2q_flow_clusters", "mpsb_update2q_flow",
    "mpsb_contract2q_batch", "mpsb_tf32_probe",
)

# CTA sizes (threads) the dataflow kernel is built for, by rows per lane
# (1: chi_cap <= 16, 2: <= 32, 4: <= 64); the first is the default.
FLOW_THREADS = {1: (64, 128), 2: (128, 256), 4: (256,)}


def rows_per_lane(chi_cap: int) -> int:
    return 1 if 2 * chi_cap <= 32 else (2 if 2 * chi_cap <= 64 else 4)


class Chain(C.Structure):
    """mpsb_chain."""
    _fields_ = [
        ("sites", C.c_void_p),
        ("bonds", C.c_void_p),
        ("norm_log", C.c_void_p),
        ("status_acc", C.c_void_p),
        ("slot_elems", C.c_int64),
        ("n", C.c_int32),
        ("chi_max", C.c_int32),
        ("cutoff", C.c_double),
    ]


class Pair(C.Structure):
    """mpsb_pair."""
    _fields_ = [("chain", C.c_int32), ("site", C.c_int32), ("gate", C.c_int32), ("out", C.c_int32)]


class FlowItem(C.Structure):
    """mpsb_flow_item."""
    _fields_ = [("chain", C.c_int32), ("site", C.c_int32), ("gate", C.c_int32), ("out", C.c_int32),
                ("dep0", C.c_int32), ("dep1", C.c_int32)]


class SiteOp(C.Structure):
    """mpsb_site_op."""
    _fields_ = [("chain", C.c_int32), ("site", C.c_int32), ("gate", C.c_int32), ("pad", C.c_int32)]


class MPSBError(RuntimeError):
    """A C-ABI call returned an error code."""


_lib = None
_lock = threading.Lock()


def _declare(lib):
    vp, i32, i64, sz, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_size_t, C.c_double
    sig = {
        "mpsb_version": (C.c_char_p, []),
        "mpsb_last_error": (C.c_char_p, []),
        "mpsb_update2q_workspace_bytes": (sz, [i32, i32]),
        "mpsb_update2q_batch": (i32, [vp, vp, i32, vp, i32, i32, dbl, i32, vp, sz, vp, vp, vp, vp, vp]),
        "mpsb_apply1q_batch": (i32, [vp, vp, i32, vp, i32, vp]),
        "mpsb_statevector": (i32, [vp, i32, i32, vp, vp, sz, vp]),
        "mpsb_amplitude": (i32, [vp, i32, i32, vp, i32, i32, vp, vp, vp]),
        "mpsb_expect_workspace_bytes": (sz, [i32, i32, i32]),
        "mpsb_expect_local": (i32, [vp, i32, i32, i32, vp, vp, vp, i32, vp, vp, sz, vp]),
        "mpsb_fp64_probe": (i32, [i64, i32, i32, vp, vp]),
        "mpsb_tf32_probe": (i32, [i64, i32, vp, vp]),
        "mpsb_contract2q_batch": (i32, [vp, vp, i32, vp, i32, i32, vp, vp, vp]),
        "mpsb_update2q_batch_noalloc": (i32, [vp, vp, i32, vp, i32, i32, dbl, i32, vp, vp, vp, vp, vp]),
        "mpsb_overlap": (i32, [vp, vp, i32, i32, vp, vp, vp, sz, vp]),
        "mpsb_update2q_tape_bytes": (sz, [i32, i32]),
        "mpsb_update2q_batch_taped": (i32, [vp, vp, i32, vp, i32, i32, dbl, i32, vp, sz, vp, sz, vp, vp, vp, vp, vp]),
        "mpsb_update2q_backward_workspace_bytes": (sz, [i32, i32]),
        "mpsb_update2q_backward_batch": (i32, [vp, vp, vp, i32, vp, i32, vp, sz, vp, vp, sz, vp, vp]),
        "mpsb_apply1q_backward_batch": (i32, [vp, vp, vp, i32, vp, i32, vp, vp]),
        "mpsb_mpo_grad_workspace_bytes": (sz, [i32, i32, i32, i32]),
        "mpsb_mpo_energy_grad": (i32, [vp, i32, i32, i32, vp, i32, vp, vp, vp, vp, sz, vp]),
        "mpsb_sample_workspace_bytes": (sz, [i32, i32]),
        "mpsb_sample": (i32, [vp, i32, i32, i32, vp, i32, vp, vp, sz, vp]),
        "mpsb_reset_batch": (i32, [vp, vp, i32, i32, vp]),
        "mpsb_canonicalize_workspace_bytes": (sz, [i32, i32]),
        "mpsb_canonicalize": (i32, [vp, vp, i32, i32, i32, i32, i32, vp, sz, vp]),
        "mpsb_update2q_flow_workspace_bytes": (sz, [i32, i32, i32, i32, i32]),
        "mpsb_update2q_flow_clusters": (i32, [i32, i32, i32]),
        "mpsb_update2q_flow": (i32, [vp, i32, vp, i32, vp, vp, vp, i32, i32, dbl, i32, i32, i32, i32, vp, sz,
                                     vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def status_text(st: int) -> str:
    """Names of the MPSB_ST_* bits set in a status word."""
    names = [(ST_NOCONV, "Jacobi not converged"), (ST_NONFINITE, "non-finite theta"),
             (ST_BADDIM, "bad bond dims"), (ST_TIMEOUT, "a bounded wait gave up"),
             (ST_CHI_LIMIT, f"an update needed a bond above {MPSB_CHI_LIMIT}")]
    return ", ".join(t for b, t in names if st & b) or "ok"


def load(path: str = LIB_PATH):
    """Load (once) and return the library handle."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise ImportError(
                    f"{path} is missing: build it with `python -m fpga_mps_simulator_b200.build` "
                    "(there is no CPU fallback)")
            lib = C.CDLL(path)
            _declare(lib)
            _lib = lib
    return _lib


class OnDevice:
    """The library handle with one CUDA device made current around every call.

    Every entry point launches on the current device (and refuses a chain
    table that lives on another one), so objects that own device memory call
    through this wrapper rather than the bare handle: a batch built on cuda:1
    then works whatever device the caller has current.
    """

    def __init__(self, lib, device):
        self._lib = lib
        self._device = device

    def __getattr__(self, name):
        fn = getattr(self._lib, name)
        if not callable(fn):
            return fn
        device = self._device

        def call(*args):
            import torch
            with torch.cuda.device(device):
                return fn(*args)

        call.__name__ = name
        return call


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().mpsb_last_error().decode(errors="replace")
        raise MPSBError(f"{what} failed ({_ERRORS.get(rc, rc)}): {msg}")


def version() -> str:
    return load().mpsb_version().decode()
