"""Pin the CPU oracle and the host gate tables to the reference's own outputs.

The golden files were produced by running the reference engine itself
(``tests/golden/make_golden.py``); these tests need no GPU.
"""
import math

import numpy as np
import pytest

from conftest import load_golden
from oracle.mps_oracle import (OracleMPS, dense_apply_1q, dense_apply_2q, dense_expect_pauli,
                               dense_to_qiskit, dense_zero_state, fidelity, haar_4x4_oracle)
from fpga_mps_simulator_b200 import gates as G
from fpga_mps_simulator_b200.circuits import brickwall, haar_4x4


def _spectra_close(log, g, rtol=1e-12):
    assert len(log) == len(g["spec_len"])
    for k, rec in enumerate(log):
        L = int(g["spec_len"][k])
        ref = g["spectra"][k, :L]
        assert rec["S"].shape[0] == L
        np.testing.assert_allclose(rec["S"], ref, rtol=0, atol=rtol * ref[0])


def test_gate_tables_match_reference():
    g = load_golden("gate_tables")
    p = list(g["params"])
    for nm, ref in zip(g["names_1q"], g["g1"]):
        np.testing.assert_allclose(G.gate_1q(str(nm), p), ref, atol=1e-15)
    for nm, ref in zip(g["names_2q"], g["g2"]):
        np.testing.assert_allclose(G.gate_2q(str(nm), p), ref, atol=1e-15)
    np.testing.assert_allclose(G.gate_2q("cnot"), G.GATE_MATRICES["cx"])


def test_haar_generator_matches_fixture_gates():
    g = load_golden("brick_n16_d10_chi16")
    ours = brickwall(16, 10, int(g["seed"]))
    assert len(ours) == len(g["sites"])
    for (i, m), si, gm in zip(ours, g["sites"], g["gates"]):
        assert i == si
        np.testing.assert_allclose(m, gm, atol=1e-15)
    rng1, rng2 = np.random.default_rng(9), np.random.default_rng(9)
    np.testing.assert_allclose(haar_4x4(rng1), haar_4x4_oracle(rng2), atol=1e-15)


@pytest.mark.parametrize("name", ["brick_n16_d10_chi16", "brick_n40_d16_chi32", "brick_n20_d12_chi64"])
def test_oracle_brickwall_matches_reference(name):
    g = load_golden(name)
    st = OracleMPS(int(g["n"]), int(g["chi_max"]), float(g["cutoff"]))
    for k, (i, gm) in enumerate(zip(g["sites"], g["gates"])):
        st.apply_adjacent_2q(int(i), gm)
        assert st.bond_dims() == list(g["bonds"][k])
        assert abs(st.norm_log - g["norm_log"][k]) <= 1e-12 * max(1.0, abs(g["norm_log"][k]))
    _spectra_close(st.log, g)
    amps = np.array([st.amplitude(b) for b in g["bits"]])
    scale = np.max(np.abs(g["amps"]))
    np.testing.assert_allclose(amps, g["amps"], rtol=0, atol=1e-11 * scale)
    if "statevector" in g:
        sv = st.statevector()
        np.testing.assert_allclose(sv, g["statevector"], rtol=0, atol=1e-12 * np.max(np.abs(sv)))


def test_oracle_xxz_matches_reference():
    g = load_golden("xxz")
    n = int(g["n"])
    st = OracleMPS(n, int(g["chi_max"]), float(g["cutoff"]))
    for i in range(n):
        st.apply_1q(i, G.gate_1q("u", [g["theta"][i], g["phi"][i], 0.0]))
    for i, gm in zip(g["sites"], g["gates"]):
        st.apply_adjacent_2q(int(i), gm)
    _spectra_close(st.log, g)
    np.testing.assert_allclose(st.norm_log, g["norm_log"][-1], rtol=1e-12)
    amps = np.array([st.amplitude(b) for b in g["bits"]])
    np.testing.assert_allclose(amps, g["amps"], rtol=0, atol=1e-11 * np.max(np.abs(g["amps"])))


def _run_diag(key, g, engine):
    n = int(g[key + "_n"])
    for kind, qa, qb, mat in zip(g[key + "_kind"], g[key + "_qa"], g[key + "_qb"], g[key + "_mat"]):
        if kind == 1:
            engine.apply_1q(int(qa), mat[:4].reshape(2, 2))
        else:
            engine.apply_2q(int(qa), int(qb), mat.reshape(4, 4))
    return n


@pytest.mark.parametrize("key", ["bell", "ghz4", "cx03", "u1", "ucxu", "ucx02", "ghz3"])
def test_oracle_diag_circuits(key):
    """fpga_diag.py:28-58 circuits: oracle == reference MPS and fidelity >= 0.999 vs exact."""
    g = load_golden("diag_circuits")
    n = int(g[key + "_n"])
    st = OracleMPS(n, 64, 1e-12)
    _run_diag(key, g, st)
    sv = st.statevector()
    np.testing.assert_allclose(sv, g[key + "_sv"], atol=1e-14)
    psi = dense_zero_state(n)
    for kind, qa, qb, mat in zip(g[key + "_kind"], g[key + "_qa"], g[key + "_qb"], g[key + "_mat"]):
        if kind == 1:
            psi = dense_apply_1q(psi, int(qa), mat[:4].reshape(2, 2))
        else:
            psi = dense_apply_2q(psi, int(qa), int(qb), mat.reshape(4, 4))
    assert fidelity(dense_to_qiskit(psi), sv) >= 0.999


def test_oracle_transfer_expectations_match_dense():
    n = 10
    st = OracleMPS(n, 64, 1e-14)
    psi = dense_zero_state(n)
    for i, gm in brickwall(n, 6, 3):
        st.apply_adjacent_2q(i, gm)
        psi = dense_apply_2q(psi, i, i + 1, gm)
    z = np.diag([1.0, -1.0]).astype(complex)
    x = G.GATE_MATRICES["x"]
    for k in range(n):
        assert abs(st.expect_local({k: z}) - dense_expect_pauli(psi, {k: z})) < 1e-12
    for k in range(n - 1):
        assert abs(st.expect_local({k: z, k + 1: z}) - dense_expect_pauli(psi, {k: z, k + 1: z})) < 1e-12
        assert abs(st.expect_local({k: x}) - dense_expect_pauli(psi, {k: x})) < 1e-12
    assert abs(st.norm_sq() - 1.0) < 1e-10


def test_oracle_ghz3_sampling():
    """GHZ-3 self-test criterion of fpga_mps_simulator.py:1147-1165."""
    g = load_golden("diag_circuits")
    st = OracleMPS(3, 16, 1e-12)
    _run_diag("ghz3", g, st)
    shots = st.sample(1024, np.random.default_rng(0))
    p = (shots.count("000") + shots.count("111")) / len(shots)
    assert p > 0.95
    ref = dict(zip(g["ghz3_count_keys"], g["ghz3_count_vals"]))
    assert sum(ref.values()) == 1024
    assert set(ref) <= {"000", "111"}


def test_oracle_truncation_rule_edge_cases():
    """keep is clipped to [1, chi_max]; a zero matrix keeps one (zero) value; norm guard."""
    st = OracleMPS(2, 1, 1e-12)
    u, sq, vh = st.svd_truncate(np.zeros((4, 4), complex))
    assert sq.shape == (1,) and sq[0] == 0.0 and st.norm_log == 0.0
    st = OracleMPS(2, 2, 1e-12)
    m = np.diag([3.0, 2.0, 1.0, 0.0]).astype(complex)
    u, sq, vh = st.svd_truncate(m)
    assert sq.shape == (2,)
    expect = 0.5 * math.log(1 - 1.0 / 14.0) + math.log(math.sqrt(13.0))
    assert abs(st.norm_log - expect) < 1e-14
    np.testing.assert_allclose(sq ** 2, np.array([3.0, 2.0]) / math.sqrt(13.0))
