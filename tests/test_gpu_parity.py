"""GPU parity of the FP64 (drop-in) two-site update against the reference.

Tolerance (FP64 form): singular values within 1e-10 * S[0] of the reference's
per-update spectrum, amplitudes within 1e-10 relative to the largest
amplitude, norm_log within 1e-10 -- the plain-form bar of the reference
engine's parity contract.  Site tensors are gauge dependent and are not
compared element-wise; amplitudes, spectra, kept counts and norm_log are.
"""
import math

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle.mps_oracle import OracleMPS, dense_apply_1q, dense_apply_2q, dense_to_qiskit, dense_zero_state
from fpga_mps_simulator_b200 import GATE_MATRICES, gate_1q
from fpga_mps_simulator_b200.circuits import brickwall_layers, haar_4x4

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _layers_from_golden(g):
    """Regroup the golden per-update (site, gate) list into brick-wall layers."""
    layers, cur, used = [], [], set()
    for i, gm in zip(g["sites"], g["gates"]):
        i = int(i)
        if i in used or i - 1 in used or i + 1 in used:
            layers.append(cur)
            cur, used = [], set()
        cur.append((i, gm))
        used.add(i)
    layers.append(cur)
    return layers


def _check_spectra(spec, kept, g, start):
    for k in range(spec.shape[0]):
        L = int(g["spec_len"][start + k])
        ref = g["spectra"][start + k, :L]
        np.testing.assert_allclose(spec[k, :L], ref, rtol=0, atol=TOL * ref[0])
        assert np.all(spec[k, L:] == 0.0)


@pytest.mark.parametrize("name", ["brick_n16_d10_chi16", "brick_n40_d16_chi32", "brick_n20_d12_chi64"])
def test_brickwall_layers_match_reference(name):
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden(name)
    n = int(g["n"])
    st = MPSState(n, int(g["chi_max"]), float(g["cutoff"]))
    done = 0
    for layer in _layers_from_golden(g):
        sites = [i for i, _ in layer]
        pb = st.apply_layer(sites, np.stack([m for _, m in layer]), record_spectra=True)
        torch.cuda.synchronize()
        assert not pb.status.any().item()
        _check_spectra(pb.spectra.cpu().numpy(), pb.kept.cpu().numpy(), g, done)
        done += len(layer)
        assert st.bond_dims() == list(g["bonds"][done - 1])
        assert abs(st.norm_log - g["norm_log"][done - 1]) <= TOL * max(1.0, abs(g["norm_log"][done - 1]))
    st.check_status()
    amps = np.array([st.amplitude(list(b)) for b in g["bits"]])
    np.testing.assert_allclose(amps, g["amps"], rtol=0, atol=TOL * np.max(np.abs(g["amps"])))
    if "statevector" in g:
        sv = st.get_statevector()
        np.testing.assert_allclose(sv, g["statevector"], rtol=0, atol=TOL * np.max(np.abs(sv)))


def test_single_update_dropin_path_matches_reference():
    """The per-update call (mps_core._apply_adjacent_2q's drop-in) on the chi=64 fixture."""
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("brick_n20_d12_chi64")
    st = MPSState(int(g["n"]), 64, float(g["cutoff"]))
    for k, (i, gm) in enumerate(zip(g["sites"], g["gates"])):
        st._apply_adjacent_2q(int(i), gm)
    torch.cuda.synchronize()
    st.check_status()
    assert st.bond_dims() == list(g["bonds"][-1])
    assert abs(st.norm_log - g["norm_log"][-1]) < TOL * abs(g["norm_log"][-1])
    amps = np.array([st.amplitude(list(b)) for b in g["bits"]])
    np.testing.assert_allclose(amps, g["amps"], rtol=0, atol=TOL * np.max(np.abs(g["amps"])))


def test_xxz_low_entanglement_matches_reference():
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("xxz")
    n = int(g["n"])
    st = MPSState(n, int(g["chi_max"]), float(g["cutoff"]))
    for i in range(n):
        st.apply_1q(i, gate_1q("u", [g["theta"][i], g["phi"][i], 0.0]))
    for i, gm in zip(g["sites"], g["gates"]):
        st._apply_adjacent_2q(int(i), gm)
    torch.cuda.synchronize()
    st.check_status()
    assert st.bond_dims() == list(g["bonds"])
    assert abs(st.norm_log - g["norm_log"][-1]) < TOL
    amps = np.array([st.amplitude(list(b)) for b in g["bits"]])
    np.testing.assert_allclose(amps, g["amps"], rtol=0, atol=TOL * np.max(np.abs(g["amps"])))


@pytest.mark.parametrize("key", ["bell", "ghz4", "cx03", "u1", "ucxu", "ucx02", "ghz3"])
def test_reference_diag_circuits(key):
    """The circuits of fpga_diag.py:28-58 and the GHZ-3 self-test, through apply_1q/apply_2q."""
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("diag_circuits")
    n = int(g[key + "_n"])
    st = MPSState(n, 64, 1e-12)
    for kind, qa, qb, mat in zip(g[key + "_kind"], g[key + "_qa"], g[key + "_qb"], g[key + "_mat"]):
        if kind == 1:
            st.apply_1q(int(qa), mat[:4].reshape(2, 2))
        else:
            st.apply_2q(int(qa), int(qb), mat.reshape(4, 4))
    sv = st.get_statevector()
    np.testing.assert_allclose(sv, g[key + "_sv"], atol=1e-12)
    if key == "ghz3":
        p = abs(sv[0]) ** 2 + abs(sv[7]) ** 2
        assert p > 0.95


def test_precision_config_full_size_against_live_oracle():
    """n=100, depth 20, chi_max=64, cutoff 1e-10: every layer in one launch."""
    from fpga_mps_simulator_b200 import MPSState
    n, depth, chi, cut = 100, 20, 64, 1e-10
    layers = brickwall_layers(n, depth, 2024)
    ref = OracleMPS(n, chi, cut)
    st = MPSState(n, chi, cut)
    for L in layers:
        pb = st.apply_layer(L.sites, L.gates, record_spectra=True)
        for i, gm in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), gm)
        spec = pb.spectra.cpu().numpy()
        for k, rec in enumerate(ref.log[-len(L.sites):]):
            S = rec["S"]
            np.testing.assert_allclose(spec[k, :len(S)], S, rtol=0, atol=TOL * S[0])
        assert list(pb.kept.cpu().numpy()) == [r["keep"] for r in ref.log[-len(L.sites):]]
    st.check_status()
    assert st.bond_dims() == ref.bond_dims()
    assert abs(st.norm_log - ref.norm_log) < TOL * abs(ref.norm_log)
    rng = np.random.default_rng(5)
    bits = rng.integers(0, 2, size=(8, n))
    amps = np.array([st.amplitude(list(b)) for b in bits])
    ref_amps = np.array([ref.amplitude(b) for b in bits])
    np.testing.assert_allclose(amps, ref_amps, rtol=1e-9, atol=0)
    z = st.expect_z_all()
    z_ref = ref.expect_z_all()
    np.testing.assert_allclose(z, z_ref, rtol=0, atol=1e-9)


def test_local_expectations_against_oracle():
    from fpga_mps_simulator_b200 import MPSState
    n = 20
    st = MPSState(n, 16, 1e-12)
    ref = OracleMPS(n, 16, 1e-12)
    for L in brickwall_layers(n, 8, 99):
        st.apply_layer(L.sites, L.gates)
        for i, gm in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), gm)
    X, Y, Z = GATE_MATRICES["x"], GATE_MATRICES["y"], GATE_MATRICES["z"]
    terms = [(k, Z, None) for k in range(n)] + [(k, X, None) for k in range(n)] + \
            [(k, Z, Z) for k in range(n - 1)] + [(k, X, Y) for k in range(n - 1)]
    got = st.expect_terms(terms)
    envs = ref.environments()
    want = [ref.expect_local({k: a} if b is None else {k: a, k + 1: b}, envs) for k, a, b in terms]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-10)
    # Pauli-string form (Qiskit order: leftmost char = qubit n-1)
    s = ["I"] * n
    s[n - 1 - 3] = "Z"
    s[n - 1 - 4] = "Z"
    assert abs(st.expectation("".join(s)) - ref.expect_local({3: Z, 4: Z})) < 1e-10


def test_apply_2q_routing_and_reversed_pairs():
    from fpga_mps_simulator_b200 import MPSState
    n = 7
    rng = np.random.default_rng(3)
    st, ref = MPSState(n, 64, 1e-12), OracleMPS(n, 64, 1e-12)
    psi = dense_zero_state(n)
    ops = [(0, 4), (5, 2), (3, 2), (1, 6), (6, 5)]
    for a, b in ops:
        gm = haar_4x4(rng)
        st.apply_2q(a, b, gm)
        ref.apply_2q(a, b, gm)
    np.testing.assert_allclose(st.get_statevector(), ref.statevector(), atol=1e-12)


def test_edge_cases_truncation_and_shapes():
    from fpga_mps_simulator_b200 import MPSState
    # chi_max = 1: every update truncates to a product state
    n = 6
    st, ref = MPSState(n, 1, 1e-12), OracleMPS(n, 1, 1e-12)
    for L in brickwall_layers(n, 4, 8):
        for i, gm in zip(L.sites, L.gates):
            st._apply_adjacent_2q(int(i), gm)
            ref.apply_adjacent_2q(int(i), gm)
    assert st.bond_dims() == [1] * (n - 1)
    assert abs(st.norm_log - ref.norm_log) < TOL
    np.testing.assert_allclose(st.get_statevector(), ref.statevector(), atol=1e-12)
    # n = 2 and odd chi caps with wide/tall thetas
    for n, chi in [(2, 64), (3, 3), (9, 7), (12, 33)]:
        st, ref = MPSState(n, chi, 1e-12), OracleMPS(n, chi, 1e-12)
        for L in brickwall_layers(n, 7, n * 31 + chi):
            st.apply_layer(L.sites, L.gates)
            for i, gm in zip(L.sites, L.gates):
                ref.apply_adjacent_2q(int(i), gm)
        st.check_status()
        assert st.bond_dims() == ref.bond_dims()
        np.testing.assert_allclose(st.get_statevector(), ref.statevector(), rtol=0,
                                   atol=TOL * np.max(np.abs(ref.statevector())))


def test_zero_gate_keeps_one_zero_value():
    """S = 0: keep is clipped to 1, nothing renormalised, the state becomes zero (mps_core.py:284-298)."""
    from fpga_mps_simulator_b200 import MPSState
    st, ref = MPSState(4, 8, 1e-12), OracleMPS(4, 8, 1e-12)
    g0 = np.zeros((4, 4), complex)
    st._apply_adjacent_2q(1, g0)
    ref.apply_adjacent_2q(1, g0)
    assert st.bond_dims() == ref.bond_dims() == [1, 1, 1]
    assert st.norm_log == ref.norm_log == 0.0
    assert np.all(st.get_statevector() == 0)


def test_nonfinite_gate_is_reported():
    from fpga_mps_simulator_b200 import MPSState
    st = MPSState(4, 8, 1e-12)
    g = np.eye(4, dtype=complex)
    g[0, 0] = np.nan
    st._apply_adjacent_2q(0, g)
    torch.cuda.synchronize()
    assert st.check_status(raise_on_error=False) & 2
    with pytest.raises(RuntimeError, match="non-finite"):
        st.check_status()


def test_bad_arguments_raise():
    from fpga_mps_simulator_b200 import MPSState
    with pytest.raises(ValueError):
        MPSState(4, 0)
    assert MPSState(4, 65).chi_max == 65  # any cap >= 1; the device limit is reported per update
    st = MPSState(6, 8)
    with pytest.raises(ValueError, match="disjoint"):
        st.apply_layer([0, 1], np.stack([np.eye(4)] * 2))
    with pytest.raises(ValueError, match="range"):
        st.apply_layer([5], np.eye(4)[None])


def test_many_chains_in_one_launch():
    from fpga_mps_simulator_b200 import MPSBatch
    specs = [(9, 4, 1e-12), (14, 16, 1e-10), (5, 64, 1e-12), (12, 8, 1e-10)]
    b = MPSBatch([s[0] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    refs = [OracleMPS(*s) for s in specs]
    per = [brickwall_layers(s[0], 6, 40 + k) for k, s in enumerate(specs)]
    for d in range(6):
        ci, si, gs = [], [], []
        for c, layers in enumerate(per):
            L = layers[d]
            ci += [c] * len(L.sites)
            si += list(L.sites)
            gs += list(L.gates)
            for i, gm in zip(L.sites, L.gates):
                refs[c].apply_adjacent_2q(int(i), gm)
        b.apply_layer(ci, si, np.stack(gs))
    b.check_status()
    for c, ref in enumerate(refs):
        assert b.bond_dims(c) == ref.bond_dims()
        assert abs(b.norm_log(c) - ref.norm_log) < TOL
        np.testing.assert_allclose(b.statevector(c), ref.statevector(), rtol=0,
                                   atol=TOL * np.max(np.abs(ref.statevector())))
