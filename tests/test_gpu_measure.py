"""GPU tests of measurement: shot sampling reproduces the reference's shots
(golden fixture from mps_core.py's own sample/get_counts) and the oracle's on
a longer chain, bit for bit, given the same seeded generator; reset matches
the reference engine's reset branch (through the oracle) including its
fall-back; through the C ABI."""
import numpy as np
import pytest

from conftest import load_golden
from oracle.mps_oracle import OracleMPS
from fpga_mps_simulator_b200.circuits import brickwall_layers

pytestmark = pytest.mark.gpu


def _pair(n, depth, chi, cut, seed):
    from fpga_mps_simulator_b200 import MPSState
    st = MPSState(n, chi, cut)
    ref = OracleMPS(n, chi, cut)
    for L in brickwall_layers(n, depth, seed):
        st.apply_layer(L.sites, L.gates)
        for i, g in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), g)
    return st, ref


def test_shots_match_reference_golden():
    g = load_golden("measure")
    st, _ = _pair(int(g["n"]), int(g["depth"]), int(g["chi_max"]), float(g["cutoff"]), int(g["seed"]))
    assert st.sample(400, rng=np.random.default_rng(11)) == list(g["shots"])
    assert st.sample(200, list(g["sub_qubits"]), np.random.default_rng(12)) == list(g["sub_shots"])
    counts = st.get_counts(300, rng=np.random.default_rng(13))
    assert sorted(counts) == list(g["count_keys"])
    assert [counts[k] for k in sorted(counts)] == list(g["count_vals"])


def test_shots_match_oracle_on_long_chain():
    st, ref = _pair(60, 12, 32, 1e-10, 5)
    a = st.sample(256, rng=np.random.default_rng(7))
    b = ref.sample(256, rng=np.random.default_rng(7))
    assert a == b


def test_zero_shots_and_bad_arguments():
    from fpga_mps_simulator_b200 import MPSState
    st = MPSState(4, 4)
    assert st.sample(0) == []
    with pytest.raises(ValueError):
        st.sample(-1)
    with pytest.raises(ValueError):
        st.reset(4)


def test_reset_matches_reference_branch():
    st, ref = _pair(8, 6, 16, 1e-12, 9)
    for site in (3, 0, 7):
        st.reset(site)
        ref.reset(site)
        sv, rv = st.get_statevector(), ref.statevector()
        np.testing.assert_allclose(sv, rv, atol=1e-12 * np.max(np.abs(rv)))


def test_reset_falls_back_to_zero_state_when_site_is_all_one():
    from fpga_mps_simulator_b200 import MPSState
    from fpga_mps_simulator_b200.gates import GATE_MATRICES
    st = MPSState(3, 4)
    ref = OracleMPS(3, 4)
    st.apply_1q(1, GATE_MATRICES["x"])
    ref.apply_1q(1, GATE_MATRICES["x"])
    st.reset(1)
    ref.reset(1)
    np.testing.assert_allclose(st.get_statevector(), ref.statevector(), atol=1e-15)
    assert abs(st.get_statevector()[0] - 1.0) < 1e-15


def _unpack(shapes, flat):
    out, k = [], 0
    for sh in shapes:
        size = int(np.prod(sh))
        out.append(flat[k:k + size].reshape(tuple(int(x) for x in sh)))
        k += size
    return out


@pytest.mark.parametrize("direction", ["left", "right"])
def test_canonical_sweeps_match_reference_elementwise(direction):
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("measure")
    sites = _unpack(g["canon_in_shapes"], g["canon_in"])
    n = len(sites)
    st = MPSState(n, 16, 1e-12)
    for k, t in enumerate(sites):
        st.sites[k] = t
    sv0 = st.get_statevector()
    if direction == "left":
        st.left_canonicalize()
        want = _unpack(g["left_shapes"], g["left"])
    else:
        st.right_canonicalize()
        want = _unpack(g["right_shapes"], g["right"])
    for k in range(n):
        got = st.sites[k]
        assert got.shape == want[k].shape
        np.testing.assert_allclose(got, want[k], atol=1e-12 * max(1.0, np.max(np.abs(want[k]))))
    np.testing.assert_allclose(st.get_statevector(), sv0, atol=1e-12 * np.max(np.abs(sv0)))


def test_single_site_normalisation_matches_oracle():
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden("measure")
    sites = _unpack(g["canon_in_shapes"], g["canon_in"])
    n = len(sites)
    st = MPSState(n, 16, 1e-12)
    ref = OracleMPS(n, 16, 1e-12)
    for k, t in enumerate(sites):
        st.sites[k] = t
    ref.sites = [t.copy() for t in sites]
    for op, i in (("l", 2), ("r", 6), ("l", 3), ("r", 1)):
        if op == "l":
            st.left_normalize_site(i)
            ref.left_normalize_site(i)
        else:
            st.right_normalize_site(i)
            ref.right_normalize_site(i)
    for k in range(n):
        np.testing.assert_allclose(st.sites[k], ref.sites[k], atol=1e-11)


def test_schmidt_values_and_entropy_match_dense_state():
    st, ref = _pair(12, 8, 64, 1e-12, 17)
    psi = ref.statevector().reshape([2] * 12)  # axis k = qubit 11 - k (Qiskit order)
    for bond in (0, 3, 5, 10):
        # qubits 0..bond on one side
        left_axes = [11 - q for q in range(bond + 1)]
        right_axes = [a for a in range(12) if a not in left_axes]
        m = np.transpose(psi, left_axes + right_axes).reshape(2 ** (bond + 1), -1)
        s = np.linalg.svd(m, compute_uv=False)
        s = s / np.linalg.norm(s)
        s = s[s > 1e-15]
        got = st.schmidt_values(bond)
        assert len(got) >= np.count_nonzero(s > 1e-12)
        np.testing.assert_allclose(got[:len(s)][s > 1e-12], s[s > 1e-12], atol=1e-12)
        p = s ** 2
        assert abs(st.exact_entanglement_entropy(bond) + float(np.sum(p * np.log(p)))) < 1e-10
