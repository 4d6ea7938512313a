"""The oracle's sampling and canonical-form restatements pinned against the
reference's own outputs (tests/golden/measure.npz, made by make_golden.py
from mps_core.py), and the uniform-threshold rule the device sampler uses
pinned against numpy's Generator.choice -- no GPU."""
import numpy as np

from conftest import load_golden
from oracle.mps_oracle import OracleMPS
from fpga_mps_simulator_b200.circuits import brickwall_layers


def _golden_state():
    g = load_golden("measure")
    n = int(g["n"])
    st = OracleMPS(n, int(g["chi_max"]), float(g["cutoff"]))
    for L in brickwall_layers(n, int(g["depth"]), int(g["seed"])):
        for i, gm in zip(L.sites, L.gates):
            st.apply_adjacent_2q(int(i), gm)
    return g, st


def _unpack(shapes, flat):
    out, k = [], 0
    for sh in shapes:
        size = int(np.prod(sh))
        out.append(flat[k:k + size].reshape(tuple(int(x) for x in sh)))
        k += size
    return out


def test_oracle_sampling_matches_reference_shots():
    g, st = _golden_state()
    assert st.sample(400, rng=np.random.default_rng(11)) == list(g["shots"])
    assert st.sample(200, list(g["sub_qubits"]), np.random.default_rng(12)) == list(g["sub_shots"])


def test_choice_equals_uniform_threshold_rule():
    """Generator.choice(2, p) draws exactly one uniform u and returns 1 iff u >= p0/(p0+p1)."""
    rng = np.random.default_rng(3)
    ps = rng.uniform(0, 1, 5000)
    a = np.random.default_rng(99)
    b = np.random.default_rng(99)
    for p in ps:
        pr = np.array([p, 1 - p])
        o = int(a.choice(2, p=pr))
        u = b.random()
        cdf0 = pr[0] / (pr[0] + pr[1])
        assert o == int(u >= cdf0)


def test_oracle_canonical_forms_match_reference():
    g = load_golden("measure")
    sites = _unpack(g["canon_in_shapes"], g["canon_in"])
    st = OracleMPS(len(sites), 64, 1e-12)
    st.sites = [t.copy() for t in sites]
    ent = [st.entanglement_entropy(b) for b in range(st.n - 1)]
    np.testing.assert_allclose(ent, g["entropy"], atol=1e-12)
    for b in range(st.n - 1):
        L = int(g["bond_spectrum_len"][b])
        np.testing.assert_allclose(st.bond_spectrum(b), g["bond_spectrum"][b, :L], atol=1e-12)
    left = st.copy()
    left.left_canonicalize()
    for got, want in zip(left.sites, _unpack(g["left_shapes"], g["left"])):
        np.testing.assert_allclose(got, want, atol=1e-12)
    right = st.copy()
    right.right_canonicalize()
    for got, want in zip(right.sites, _unpack(g["right_shapes"], g["right"])):
        np.testing.assert_allclose(got, want, atol=1e-12)
