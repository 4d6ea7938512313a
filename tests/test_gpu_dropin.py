"""The drop-in class against what a user of the reference class sees.

* ``MPSState(n)`` keeps the reference's defaults (chi_max = 256, svd_cutoff =
  1e-12, mps_core.py:185): a 12-qubit circuit (bonds stay within 64) matches
  the reference's amplitudes, bonds and norm_log; a 14-qubit one whose middle
  bond needs 128 is refused at read-out (MPSB_ST_CHI_LIMIT) instead of
  returning a differently truncated state.
* ``entanglement_entropy`` and ``bond_spectrum`` follow mps_core.py:465-494 in
  the reference's own (non-canonical) gauge; ``exact_entanglement_entropy``
  is the gauge-independent one.
* The C ABI refuses a chain table that is not device memory of the current
  device instead of launching on it.

Tolerances: amplitudes and spectra within 1e-10 (relative to the largest
value), entropies within 1e-10 absolute -- the plain form's parity bar.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _run(st, sites, gates):
    for i, g in zip(sites, gates):
        st.apply_2q(int(i), int(i) + 1, g)


def test_default_chi_max_matches_reference_within_device_limit():
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("dropin")
    st = MPSState(12)
    assert st.chi_max == int(g["d12_chi_max"]) == 256 and st.svd_cutoff == float(g["d12_cutoff"])
    _run(st, g["d12_sites"], g["d12_gates"])
    assert st.bond_dims() == [int(v) for v in g["d12_bonds"]] and st.max_bond() == 64
    assert abs(st.norm_log - float(g["d12_norm_log"])) < TOL
    bits = g["d12_bits"].astype(np.uint8)
    got = np.array([st.amplitude(list(b)) for b in bits])
    np.testing.assert_allclose(got, g["d12_amps"], rtol=0, atol=TOL * np.abs(g["d12_amps"]).max())


def test_bond_above_device_limit_is_refused_not_silently_truncated():
    from fpga_mps_simulator_b200 import MPSState, _lib
    g = load_golden("dropin")
    assert int(g["d14_bonds"].max()) > _lib.MPSB_CHI_LIMIT  # the reference forms a 128 bond
    st = MPSState(14)
    _run(st, g["d14_sites"], g["d14_gates"])
    torch.cuda.synchronize()
    assert st.check_status(raise_on_error=False) & _lib.ST_CHI_LIMIT
    with pytest.raises(RuntimeError, match="bond above 64"):
        st.get_statevector()
    with pytest.raises(RuntimeError, match="chi_max <= 64"):
        st.amplitude([0] * 14)
    # with the cap stated explicitly the same circuit runs and truncates at 64
    st64 = MPSState(14, chi_max=64)
    _run(st64, g["d14_sites"], g["d14_gates"])
    assert st64.check_status() == 0 and st64.max_bond() == 64


@pytest.mark.parametrize("key,chi,cut", [("b16", 16, 1e-12), ("b20", 64, 1e-10)])
def test_entropy_and_bond_spectrum_follow_reference_gauge(key, chi, cut):
    from fpga_mps_simulator_b200 import MPSState
    from fpga_mps_simulator_b200.circuits import brickwall_layers
    g = load_golden("dropin")
    n = {"b16": 16, "b20": 20}[key]
    depth, seed = {"b16": (10, 1234), "b20": (12, 4242)}[key]
    st = MPSState(n, chi, cut)
    for L in brickwall_layers(n, depth, seed):
        st.apply_layer(L.sites, L.gates)
    assert st.bond_dims() == [int(v) for v in g[key + "_bonds"]]
    ent = np.array([st.entanglement_entropy(b) for b in range(n - 1)])
    np.testing.assert_allclose(ent, g[key + "_entropy"], rtol=0, atol=TOL)
    for b in range(n):
        L = int(g[key + "_bond_spectrum_len"][b])
        got = st.bond_spectrum(b)
        assert len(got) == L, (b, len(got), L)
        np.testing.assert_allclose(got, g[key + "_bond_spectrum"][b, :L], rtol=0, atol=TOL)
    # the reference-gauge entropy differs from the exact one on this non-canonical state
    exact = np.array([st.exact_entanglement_entropy(b) for b in range(n - 1)])
    assert np.max(np.abs(exact - ent)) > 1e-3
    # a mixed-canonical copy at bond b makes the two agree (the reference's premise)
    b = n // 2
    m = st.copy()
    m._b.canonicalize([0], b + 1, n - 1, "right")
    assert abs(m.entanglement_entropy(b) - st.exact_entanglement_entropy(b)) < 1e-9


def test_deferred_gate_by_gate_calls_equal_eager_calls_bitwise():
    """The drop-in queues _apply_adjacent_2q / apply_2q calls and runs them as one
    dataflow launch at the next read; the state must be exactly what one launch per
    call gives -- with SWAP routing, reversed pairs and single-site gates in between
    (each of which flushes the queue first)."""
    from fpga_mps_simulator_b200 import MPSState, gate_1q
    from fpga_mps_simulator_b200.circuits import haar_4x4
    rng = np.random.default_rng(17)
    n = 10
    ops = []
    for _ in range(60):
        r = rng.random()
        if r < 0.7:
            i = int(rng.integers(0, n - 1))
            ops.append(("2", i, i + 1, haar_4x4(rng)))
        elif r < 0.8:
            i, j = (int(v) for v in rng.choice(n, 2, replace=False))
            ops.append(("2", i, j, haar_4x4(rng)))  # routed or reversed
        else:
            ops.append(("1", int(rng.integers(0, n)), gate_1q("u", list(rng.uniform(-3, 3, 3)))))
    ops.append(("2", 3, 4, haar_4x4(rng)))  # end on a two-site gate: it stays queued until the read
    states = {}
    for defer in (True, False):
        st = MPSState(n, 16, 1e-12, defer=defer)
        for op in ops:
            if op[0] == "2":
                st.apply_2q(op[1], op[2], op[3])
            else:
                st.apply_1q(op[1], op[2])
        states[defer] = st
    d, e = states[True], states[False]
    assert len(d._pending) > 0  # the last calls are still queued; reading _b below flushes them
    for x, y in zip(d._b.snapshot(), e._b.snapshot()):
        assert torch.equal(x, y)
    assert d.last_flow is not None and d.norm_log == e.norm_log
    with pytest.raises(ValueError, match="range"):
        d._apply_adjacent_2q(n - 1, np.eye(4))


def test_chain_table_in_host_memory_is_refused():
    from fpga_mps_simulator_b200 import MPSBatch, _lib
    b = MPSBatch([4], 4, 1e-12)
    pb = b.make_pairs([0], [1], np.eye(4, dtype=np.complex128)[None])
    lib = _lib.load()
    host_table = (C.c_uint8 * b.table.numel())(*b.table.cpu().numpy().tolist())
    ws = torch.empty(lib.mpsb_update2q_workspace_bytes(1, b.chi_cap), dtype=torch.uint8, device=b.device)
    rc = lib.mpsb_update2q_batch(C.addressof(host_table), pb.pairs.data_ptr(), 1, pb.gates.data_ptr(), _lib.FP64,
                                 b.chi_cap, 0.0, 0, ws.data_ptr(), ws.numel(), None, pb.kept.data_ptr(),
                                 pb.trunc.data_ptr(), pb.status.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == -1 and b"not device memory" in lib.mpsb_last_error()
    torch.cuda.synchronize()  # nothing was launched, the context is intact
    b.run_pairs(pb)
    torch.cuda.synchronize()
    assert b.check_status() == 0
