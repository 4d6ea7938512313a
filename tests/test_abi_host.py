"""CPU-side checks: the C-ABI library loads and exports every declared symbol,
host-only entry points behave, and the host logic around the kernels is right.
No GPU compute is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from fpga_mps_simulator_b200 import _lib, gates as G
from fpga_mps_simulator_b200.mps import validate_pairs

HEADER = os.path.join(ROOT, "include", "mpsb200.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"MPSB_API\s+[\w\s\*]*?\b(mpsb_\w+)\s*\(", txt)))


def test_header_declares_the_binding_exports():
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert "sm_100a" in _lib.version()


def test_struct_sizes_match_header_layout():
    # mpsb_chain: 4 pointers, int64, 2 x int32, double
    assert C.sizeof(_lib.Chain) == 4 * 8 + 8 + 8 + 8
    assert C.sizeof(_lib.Pair) == 16 and C.sizeof(_lib.SiteOp) == 16


def test_workspace_sizes():
    lib = _lib.load()
    assert lib.mpsb_update2q_workspace_bytes(10, 65) == 0
    assert lib.mpsb_update2q_workspace_bytes(-1, 8) == 0
    w1 = lib.mpsb_update2q_workspace_bytes(1, 64)
    w2 = lib.mpsb_update2q_workspace_bytes(2, 64)
    assert w2 - w1 >= 128 * 128 * 16


def test_argument_errors_need_no_device():
    lib = _lib.load()
    assert lib.mpsb_update2q_batch(None, None, 0, None, 0, 8, 0.0, 0, None, 0, None, None, None, None, None) == 0
    rc = lib.mpsb_update2q_batch(None, None, -1, None, 0, 8, 0.0, 0, None, 0, None, None, None, None, None)
    assert rc == -1 and b"npairs" in lib.mpsb_last_error()
    rc = lib.mpsb_update2q_batch(C.c_void_p(256), C.c_void_p(256), 1, C.c_void_p(256), 0, 99, 0.0, 0,
                                 C.c_void_p(256), 1 << 30, None, None, None, C.c_void_p(256), None)
    assert rc == -1 and b"chi_cap" in lib.mpsb_last_error()
    rc = lib.mpsb_update2q_batch(C.c_void_p(256), C.c_void_p(256), 1, C.c_void_p(256), 7, 8, 0.0, 0,
                                 C.c_void_p(256), 1 << 30, None, None, None, C.c_void_p(256), None)
    assert rc == -1 and b"precision" in lib.mpsb_last_error()
    rc = lib.mpsb_update2q_batch(C.c_void_p(256), C.c_void_p(256), 4, C.c_void_p(256), 0, 8, 0.0, 0,
                                 C.c_void_p(256), 16, None, None, None, C.c_void_p(256), None)
    assert rc == -3
    with pytest.raises(_lib.MPSBError, match="EINVAL"):
        _lib.check(-1, "probe")
    # contraction only: same argument rules, checked before any device query
    p = C.c_void_p(256)
    assert lib.mpsb_contract2q_batch(None, None, 0, None, 0, 8, None, None, None) == 0
    rc = lib.mpsb_contract2q_batch(p, p, -2, p, 0, 8, p, p, None)
    assert rc == -1 and b"npairs" in lib.mpsb_last_error()
    rc = lib.mpsb_contract2q_batch(p, p, 1, p, 0, 8, None, p, None)
    assert rc == -1 and b"theta" in lib.mpsb_last_error()
    rc = lib.mpsb_contract2q_batch(p, p, 1, p, 0, 65, p, p, None)
    assert rc == -1 and b"chi_cap" in lib.mpsb_last_error()
    rc = lib.mpsb_contract2q_batch(p, p, 1, p, 3, 8, p, p, None)
    assert rc == -1 and b"precision" in lib.mpsb_last_error()
    # the TF32 probe bounds its MMA chain
    assert lib.mpsb_tf32_probe(0, 1, p, None) == -1
    assert lib.mpsb_tf32_probe(65537, 1, p, None) == -1
    assert lib.mpsb_tf32_probe(1024, 0, p, None) == -1


def test_keep_limit_and_status_names():
    # min(chi_max, the device limit 64, the Schmidt bound 2^(n//2) of an n-site chain)
    assert _lib.keep_limit(12, 256) == 64 and _lib.keep_limit(8, 256) == 16
    assert _lib.keep_limit(100, 32) == 32 and _lib.keep_limit(1, 256) == 1 and _lib.keep_limit(5, 3) == 3
    assert _lib.status_text(0) == "ok"
    assert "bond above 64" in _lib.status_text(_lib.ST_CHI_LIMIT | _lib.ST_NOCONV)
    hdr = open(HEADER).read()
    assert re.search(r"MPSB_ST_CHI_LIMIT\s*=\s*16", hdr) and re.search(r"MPSB_ST_TIMEOUT\s*=\s*8", hdr)


def test_library_calls_run_with_the_owner_device_current(monkeypatch):
    # every entry point launches on the current device, so a batch on cuda:1
    # must make cuda:1 current around each call, whatever the caller has current
    import torch
    seen = []

    class Ctx:
        def __init__(self, d):
            self.d = d

        def __enter__(self):
            seen.append(("enter", self.d))

        def __exit__(self, *exc):
            seen.append(("exit", self.d))

    class FakeLib:
        version = "not a call"

        def mpsb_probe(self, x):
            seen.append(("call", x))
            return 7

    monkeypatch.setattr(torch.cuda, "device", Ctx)
    lib = _lib.OnDevice(FakeLib(), "cuda:1")
    assert lib.mpsb_probe(3) == 7
    assert seen == [("enter", "cuda:1"), ("call", 3), ("exit", "cuda:1")]
    assert lib.version == "not a call"


def test_validate_pairs():
    validate_pairs([10], [0, 0, 0], [0, 2, 8])
    validate_pairs([10, 6], [0, 0, 1, 1], [1, 5, 0, 4])
    with pytest.raises(ValueError, match="disjoint"):
        validate_pairs([10], [0, 0], [2, 3])
    with pytest.raises(ValueError, match="range"):
        validate_pairs([10], [0], [9])
    with pytest.raises(ValueError, match="contiguous"):
        validate_pairs([10, 10], [0, 1, 0], [0, 0, 4])
    with pytest.raises(ValueError, match="range"):
        validate_pairs([10], [1], [0])


def test_permute_and_route_match_reference_dispatch():
    g = np.arange(16).reshape(4, 4).astype(complex)
    p = G.permute_2q(g)
    # |ab> -> |ba>: row/col 1 <-> 2
    assert p[1, 2] == g[2, 1] and p[0, 3] == g[0, 3] and p[2, 2] == g[1, 1]
    route = G.swap_route(5, 1, "cx")
    assert route == [("swap", [4, 5], None), ("swap", [3, 4], None), ("swap", [2, 3], None),
                     ("cx", [1, 2], None), ("swap", [2, 3], None), ("swap", [3, 4], None),
                     ("swap", [4, 5], None)]
