"""GPU parity of the contraction-only entry point (mpsb_contract2q_batch).

theta = G (A B) as the (2 chi_l) x (2 chi_r) matrix the reference's FPGA
kernel writes for its host SVD (fpga_mps_simulator.cpp:287-371,
fpga_mps_simulator.py:584-600), checked against the oracle's einsum
(mps_core.py:334-340):

* FP64: within 1e-12 of max |theta| (summation order differs from numpy's),
  and bitwise equal to the matrix the FP64 update itself factorises (read
  from its adjoint tape);
* 3xTF32 tensor-core forms: within 5e-6 of max |theta| (about twenty times the
  ~2.4e-7 relative rounding of a 3xTF32 product summed over chi_m terms,
  with the complex-3M cancellation).
"""

import numpy as np
import pytest
import torch

from oracle.mps_oracle import OracleMPS

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-12
TF32_TOL = 5e-6


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)


def _haar(rng):
    q, r = np.linalg.qr(_rand(rng, (4, 4)))
    return q * (np.diag(r) / np.abs(np.diag(r)))[None, :]


def _oracle_theta(A, B, G):
    cl, cr = A.shape[0], B.shape[2]
    t = np.einsum("lpm,mqr->lpqr", A, B).reshape(cl, 4, cr)
    return np.einsum("st,ltr->lsr", G, t).reshape(2 * cl, 2 * cr)


def _batch_with_pair(cl, cm, cr, chi, rng, n=16, i=7):
    from fpga_mps_simulator_b200 import MPSBatch
    b = MPSBatch([n], [chi], [1e-12])
    A, B = _rand(rng, (cl, 2, cm)), _rand(rng, (cm, 2, cr))
    b.set_site(0, i, A)
    b.set_site(0, i + 1, B)
    return b, A, B


SHAPES = [
    (1, 1, 1, 4),      # product state
    (1, 2, 2, 4),      # chain end
    (4, 8, 4, 64),     # square, small
    (8, 8, 2, 64),     # tall
    (2, 8, 8, 64),     # wide (the update would factorise theta^H)
    (13, 7, 9, 16),    # odd sizes
    (32, 32, 32, 32),  # saturated chi = 32
    (40, 32, 45, 64),  # ragged at chi_cap 64
    (64, 64, 64, 64),  # saturated chi = 64: 128 x 128 theta
]


@pytest.mark.parametrize("cl,cm,cr,chi", SHAPES)
def test_fp64_theta_matches_oracle(cl, cm, cr, chi):
    rng = np.random.default_rng(cl * 1000 + cm * 10 + cr)
    b, A, B = _batch_with_pair(cl, cm, cr, chi, rng)
    G = _haar(rng) + 0.25 * _rand(rng, (4, 4))  # general (non-unitary) gate
    got = b.thetas([0], [7], G[None], precision="fp64")[0]
    want = _oracle_theta(A, B, G)
    assert got.shape == want.shape == (2 * cl, 2 * cr)
    assert np.max(np.abs(got - want)) <= FP64_TOL * np.max(np.abs(want))


@pytest.mark.parametrize("precision,chi", [("mixed", 64), ("mixed_all", 64), ("mixed_all", 32),
                                           ("mixed_all", 16)])
@pytest.mark.parametrize("shape", ["square", "tall", "wide"])
def test_tensor_core_theta_close_to_oracle(precision, chi, shape):
    c = chi
    cl, cm, cr = {"square": (c, c, c), "tall": (c, c, max(1, c // 4)), "wide": (max(1, c // 2), c, c)}[shape]
    rng = np.random.default_rng(chi + len(shape))
    b, A, B = _batch_with_pair(cl, cm, cr, chi, rng)
    G = _haar(rng)
    got = b.thetas([0], [7], G[None], precision=precision)[0]
    want = _oracle_theta(A, B, G)
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err <= TF32_TOL, err
    assert err > 0.0  # the tensor-core form really ran (the FP64 one would agree to ~1e-16)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("cl,cm,cr", [(64, 64, 64), (64, 48, 40), (24, 64, 64)])
def test_theta_is_the_matrix_the_update_factorises(precision, cl, cm, cr):
    """Bitwise: the update's adjoint tape starts with X = theta (theta^H when wide)."""
    from fpga_mps_simulator_b200.adjoint import AdjointEngine, Step2Q
    from fpga_mps_simulator_b200.hamiltonians import zz_mpo
    rng = np.random.default_rng(cl + 3 * cm + 7 * cr)
    b, A, B = _batch_with_pair(cl, cm, cr, 64, rng)
    b.precision = precision
    G = _haar(rng)
    th = b.thetas([0], [7], G[None], precision=precision)[0]
    eng = AdjointEngine(b, zz_mpo(16))
    pb = b.make_pairs([0], [7], G[None])
    rec = eng._record(Step2Q(pb, b.chi_cap))
    torch.cuda.synchronize()
    assert int(pb.status.item()) == 0
    trans = cr > cl
    R, C = (2 * cr, 2 * cl) if trans else (2 * cl, 2 * cr)
    X = rec[2].view(torch.complex128)[: R * C].cpu().numpy().reshape(R, C)
    if trans:
        # the FP64 loop conjugates the same products; the tensor-core GEMM swaps
        # operand roles, which reorders its fp32 accumulation
        if precision == "fp64":
            assert np.array_equal(X, th.conj().T)
        else:
            assert np.max(np.abs(X - th.conj().T)) <= TF32_TOL * np.max(np.abs(th))
    else:
        assert np.array_equal(X, th)


def test_many_overlapping_pairs_in_one_launch():
    """Pairs only read the sites: every adjacent pair of a state at once."""
    from fpga_mps_simulator_b200 import MPSState
    from fpga_mps_simulator_b200.circuits import brickwall_layers
    n, chi = 14, 16
    st = MPSState(n, chi, 1e-12)
    ref = OracleMPS(n, chi, 1e-12)
    for L in brickwall_layers(n, 6, 11):
        st.apply_layer(L.sites, L.gates)
        for i, g in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), g)
    rng = np.random.default_rng(5)
    gates = np.stack([_haar(rng) for _ in range(n - 1)])
    bonds_before = st.bond_dims()
    got = st._b.thetas(np.zeros(n - 1, np.int32), np.arange(n - 1), gates)
    assert st.bond_dims() == bonds_before
    # theta is gauge dependent, so compare the gauge-invariant singular values
    for i in range(n - 1):
        want = _oracle_theta(ref.sites[i], ref.sites[i + 1], gates[i])
        s_got, s_want = np.linalg.svd(got[i], compute_uv=False), np.linalg.svd(want, compute_uv=False)
        np.testing.assert_allclose(s_got, s_want, rtol=0, atol=1e-10 * s_want[0])


def test_mpsstate_theta_leaves_the_state_alone():
    from fpga_mps_simulator_b200 import MPSState
    rng = np.random.default_rng(3)
    st = MPSState(6, 8, 1e-12)
    for i in (0, 2, 4, 1, 3):
        st.apply_2q(i, i + 1, _haar(rng))
    psi = st.get_statevector()
    G = _haar(rng)
    th = st.theta(2, G)
    A, B = st.sites[2], st.sites[3]
    assert np.max(np.abs(th - _oracle_theta(A, B, G))) <= FP64_TOL * np.max(np.abs(th))
    np.testing.assert_array_equal(st.get_statevector(), psi)
    with pytest.raises(ValueError):
        st.theta(5, G)


def test_bad_bond_dims_flagged_per_pair():
    from fpga_mps_simulator_b200 import MPSBatch
    b = MPSBatch([8], [4], [1e-12])
    rng = np.random.default_rng(1)
    tb = b.make_thetas([0, 0], [2, 4], np.stack([_haar(rng), _haar(rng)]))
    saved = b.bonds.clone()
    b.bonds[int(b.bond_off[0]) + 5] = b.chi_cap + 1  # the middle bond of pair (4, 5)
    b.run_thetas(tb)
    torch.cuda.synchronize()
    b.bonds.copy_(saved)
    from fpga_mps_simulator_b200 import _lib
    assert tb.status.cpu().tolist() == [0, _lib.ST_BADDIM]


def test_tf32_probe_counts_and_rate():
    from fpga_mps_simulator_b200 import _lib
    lib = _lib.load()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    sink = torch.zeros(sms, dtype=torch.float64, device="cuda")
    iters = 4096
    stream = torch.cuda.current_stream()
    _lib.check(lib.mpsb_tf32_probe(iters, sms, sink.data_ptr(), stream.cuda_stream), "tf32 probe")
    torch.cuda.synchronize()
    # every accumulator element: iters * K products of tf32(1/64) * tf32(1/128), exact in fp32
    assert torch.all(sink == iters * 8 / 8192.0).item()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _lib.check(lib.mpsb_tf32_probe(iters, sms, sink.data_ptr(), stream.cuda_stream), "tf32 probe")
    e1.record(stream)
    torch.cuda.synchronize()
    tflops = 2.0 * 128 * 256 * 8 * iters * sms / (e0.elapsed_time(e1) * 1e-3) / 1e12
    assert tflops > 100.0, tflops  # a dense tensor-core rate, not a fallback
    with pytest.raises(RuntimeError):
        _lib.check(lib.mpsb_tf32_probe(1 << 20, sms, sink.data_ptr(), stream.cuda_stream), "tf32 probe")


def test_pairs_of_many_chains_and_graph_replay():
    """Pairs of uneven chains in one launch; the launch captured in a CUDA graph
    and replayed gives the same thetas bit for bit."""
    from fpga_mps_simulator_b200 import MPSBatch
    from fpga_mps_simulator_b200.circuits import brickwall_layers
    ns = [6, 11, 9]
    b = MPSBatch(ns, [8, 16, 4], [1e-12] * 3)
    refs = [OracleMPS(n, chi, 1e-12) for n, chi in zip(ns, [8, 16, 4])]
    for c, n in enumerate(ns):
        for L in brickwall_layers(n, 5, 20 + c):
            b.apply_layer(np.full(len(L.sites), c, np.int32), L.sites, L.gates)
            for i, g in zip(L.sites, L.gates):
                refs[c].apply_adjacent_2q(int(i), g)
    rng = np.random.default_rng(9)
    chain_idx = np.array([0, 2, 1, 1, 0, 2], np.int32)
    sites = np.array([2, 0, 5, 9, 4, 7], np.int32)
    gates = np.stack([_haar(rng) for _ in sites])
    tb = b.make_thetas(chain_idx, sites, gates)
    b.run_thetas(tb)
    torch.cuda.synchronize()
    assert not tb.status.any().item()
    first = tb.theta.clone()
    for k, (c, i) in enumerate(zip(chain_idx, sites)):
        want = _oracle_theta(refs[c].sites[i], refs[c].sites[i + 1], gates[k])
        got = tb.matrices()[k]
        s_got, s_want = np.linalg.svd(got, compute_uv=False), np.linalg.svd(want, compute_uv=False)
        np.testing.assert_allclose(s_got, s_want, rtol=0, atol=1e-10 * s_want[0])
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    tb.theta.zero_()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        b.run_thetas(tb, stream=s)
    for _ in range(2):
        tb.theta.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(tb.theta, first)
    del g
