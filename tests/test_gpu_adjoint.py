"""GPU tests of the hand-written adjoint, checked against the CPU adjoint of
oracle/mps_adjoint.py (itself pinned by finite differences and parameter
shift in test_adjoint_oracle.py), against device parameter-shift and central
finite differences of the device forward, and across its own modes
(checkpointed vs taped, autograd.Function vs direct)."""
import math

import numpy as np
import pytest
import torch

from oracle.mps_adjoint import (apply1q_backward, hea_energy_grad, mpo_energy_grad, tfim_mpo as oracle_tfim,
                                update_backward_given_outputs, update_forward)

pytestmark = pytest.mark.gpu
REL = 1e-9


def _rand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _haar(rng):
    q, r = np.linalg.qr(_rand(rng, (4, 4)))
    return q * (np.diag(r) / np.abs(np.diag(r)))[None, :]


def _slot(b, k):
    return int(b.site_off[0]) + k


def _put_cot(b, cot, k, arr):
    row = torch.zeros(b.slot, dtype=torch.complex128)
    row[: arr.size] = torch.from_numpy(np.ascontiguousarray(arr).reshape(-1))
    cot[_slot(b, k)].copy_(row.to(b.device))


def _get(t, b, k, shape):
    return t[_slot(b, k), : int(np.prod(shape))].cpu().numpy().reshape(shape)


@pytest.mark.parametrize("cl,cm,cr,chi,cut,gate_kind,graded", [
    (4, 8, 4, 64, 1e-12, "haar", False),      # square, no truncation
    (8, 8, 2, 64, 1e-12, "haar", False),      # tall theta (Jacobi on theta)
    (2, 8, 8, 64, 1e-12, "haar", False),      # wide theta (Jacobi on theta^H)
    (4, 4, 4, 4, 1e-12, "haar", False),       # chi truncation with kept/discarded coupling
    (16, 16, 16, 16, 1e-12, "general", False),  # non-unitary gate, truncation
    (32, 32, 32, 32, 1e-12, "haar", False),   # chi = 32 saturated layer shape
    (64, 64, 64, 64, 1e-10, "haar", False),   # chi = 64, 128 x 128 theta
    # graded theta: the QR-preconditioned path (Jacobi on R^H, right-side tape)
    (16, 16, 16, 16, 1e-12, "haar", True),
    (32, 32, 32, 32, 1e-12, "general", True),
    (64, 64, 64, 64, 1e-10, "haar", True),
    (12, 16, 24, 32, 1e-12, "haar", True),    # wide: preconditioned Jacobi on theta^H
    (20, 16, 13, 32, 1e-12, "haar", True),    # tall, C = 26: the last QR panel half padding
    (24, 24, 24, 32, 1e-12, "haar", True),    # C_pad = 48: two quads on some warps, one on others
    (40, 32, 45, 64, 1e-12, "general", True),  # wide, C = 80 at chi_cap 64
    (4, 8, 4, 64, 1e-12, "haar", True),       # too few columns for the preconditioner
])
def test_update_backward_matches_oracle(cl, cm, cr, chi, cut, gate_kind, graded):
    from fpga_mps_simulator_b200 import MPSBatch, _lib
    from fpga_mps_simulator_b200.adjoint import AdjointEngine, Step2Q
    from fpga_mps_simulator_b200.hamiltonians import zz_mpo
    rng = np.random.default_rng(cl * 1000 + cm * 10 + cr + 7 * graded)
    n, i = 16, 7
    b = MPSBatch([n], [chi], [cut])
    A, B = _rand(rng, (cl, 2, cm)), _rand(rng, (cm, 2, cr))
    if graded:  # column norms of theta (and of theta^H) spread over ~3 decades
        A *= np.logspace(0.0, -1.5, cl)[:, None, None]
        B *= np.logspace(0.0, -1.5, cr)[None, None, :]
    G = _haar(rng) if gate_kind == "haar" else _haar(rng) + 0.3 * _rand(rng, (4, 4))
    b.set_site(0, i, A)
    b.set_site(0, i + 1, B)
    eng = AdjointEngine(b, zz_mpo(n))
    pb = b.make_pairs([0], [i], G[None])
    step = Step2Q(pb, b.chi_cap)
    rec = eng._record(step)
    torch.cuda.synchronize()
    assert int(pb.status.item()) == 0
    # tape side flag (meta double 132): set exactly when the pair was preconditioned
    q = (2 * b.chi_cap) ** 2
    side = float(rec[2].view(torch.float64)[4 * q + 132].item())
    assert side == (1.0 if graded and 2 * min(cl, cr) > 16 else 0.0), side
    k = int(pb.kept.item())
    Ap, Bp = b.site(0, i), b.site(0, i + 1)
    # forward parity on the gauge-invariant product A' B' and the kept count
    rAp, rBp, aux = update_forward(A, B, G, chi, cut)
    assert k == aux["keep"]
    got_t = np.einsum("lpm,mqr->lpqr", Ap, Bp)
    want_t = np.einsum("lpm,mqr->lpqr", rAp, rBp)
    assert np.max(np.abs(got_t - want_t)) <= 1e-10 * max(1.0, np.max(np.abs(want_t)))
    Cb_a, Cb_b = _rand(rng, (cl, 2, k)), _rand(rng, (k, 2, cr))
    eng.cot.zero_()
    _put_cot(b, eng.cot, i, Cb_a)
    _put_cot(b, eng.cot, i + 1, Cb_b)
    # the backward with the gate cotangent, through the C ABI
    lib = _lib.load()
    pre_table = b.make_table(*rec[1])
    gg = torch.zeros(1, 16, dtype=torch.complex128, device=b.device)
    status = torch.zeros(1, dtype=torch.int32, device=b.device)
    need = lib.mpsb_update2q_backward_workspace_bytes(1, b.chi_cap)
    ws = torch.empty(need, dtype=torch.uint8, device=b.device)
    rc = lib.mpsb_update2q_backward_batch(pre_table.data_ptr(), eng.cot_table.data_ptr(), pb.pairs.data_ptr(), 1,
                                          pb.gates.data_ptr(), b.chi_cap, rec[2].data_ptr(), rec[2].numel(),
                                          gg.data_ptr(), ws.data_ptr(), ws.numel(), status.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "backward")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    Ab, Bb = _get(eng.cot, b, i, (cl, 2, cm)), _get(eng.cot, b, i + 1, (cm, 2, cr))
    rA, rB, rG = update_backward_given_outputs(A, B, G, Ap, Bp, Cb_a, Cb_b, need_gate=True)
    for got, want in ((Ab, rA), (Bb, rB), (gg.cpu().numpy().reshape(4, 4), rG)):
        assert np.max(np.abs(got - want)) <= REL * 1e3 * max(1.0, np.max(np.abs(want))), np.max(np.abs(got - want))


def test_apply1q_backward_matches_oracle():
    from fpga_mps_simulator_b200 import MPSBatch, _lib
    rng = np.random.default_rng(4)
    n = 8
    b = MPSBatch([n], [8], [1e-12])
    A = _rand(rng, (4, 2, 8))
    b.set_site(0, 3, A)
    G = _rand(rng, (2, 2))
    cot = torch.zeros_like(b.sites)
    C = _rand(rng, (4, 2, 8))
    _put_cot(b, cot, 3, C)
    ops = torch.tensor([[0, 3, 0, 0]], dtype=torch.int32, device=b.device)
    g = torch.from_numpy(G.reshape(1, 4)).to(b.device)
    gg = torch.zeros(1, 4, dtype=torch.complex128, device=b.device)
    lib = _lib.load()
    rc = lib.mpsb_apply1q_backward_batch(b.table.data_ptr(), b.make_table(cot, b.bonds).data_ptr(), ops.data_ptr(),
                                         1, g.data_ptr(), b.chi_cap, gg.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "apply1q backward")
    rA, rG = apply1q_backward(A, G, C)
    np.testing.assert_allclose(_get(cot, b, 3, A.shape), rA, atol=1e-12)
    np.testing.assert_allclose(gg.cpu().numpy().reshape(2, 2), rG, atol=1e-11)


def test_mpo_energy_and_site_cotangents_match_oracle():
    from fpga_mps_simulator_b200 import MPSBatch
    from fpga_mps_simulator_b200.adjoint import AdjointEngine
    from fpga_mps_simulator_b200.hamiltonians import tfim_mpo
    rng = np.random.default_rng(8)
    n, bonds = 7, [1, 2, 4, 5, 4, 3, 2, 1]
    b = MPSBatch([n, n], [8, 8], [1e-12, 1e-12])
    sites = [[_rand(rng, (bonds[k], 2, bonds[k + 1])) for k in range(n)] for _ in range(2)]
    for c in range(2):
        for k in range(n):
            b.set_site(c, k, sites[c][k])
    eng = AdjointEngine(b, tfim_mpo(n, 1.0, 0.8))
    w = torch.tensor([1.0, -0.5], dtype=torch.float64, device=b.device)
    loss = eng.energy(w).cpu().numpy()
    for c in range(2):
        L, cots = mpo_energy_grad(sites[c], oracle_tfim(n, 1.0, 0.8))
        assert abs(loss[c] - L) < 1e-11
        for k in range(n):
            got = eng.cot[int(b.site_off[c]) + k, : cots[k].size].cpu().numpy().reshape(cots[k].shape)
            np.testing.assert_allclose(got, float(w[c]) * cots[k], atol=1e-10 * max(1.0, np.max(np.abs(cots[k]))))


def test_hea_gradient_matches_oracle_and_parameter_shift():
    from fpga_mps_simulator_b200.adjoint import HEAEnergy
    n, layers, nvec = 8, 2, 3
    rng = np.random.default_rng(21)
    angles = rng.uniform(0, 2 * np.pi, (nvec, layers, n, 2))
    model = HEAEnergy(n, layers, nvec, chi_max=16, cutoff=1e-12)
    e, g = model.energy_and_grad(angles)
    e, g = e.cpu().numpy(), g.cpu().numpy()
    for c in range(nvec):
        L, G = hea_energy_grad(angles[c], oracle_tfim(n), 16, 1e-12)
        assert abs(e[c] - L) < 1e-10
        assert np.max(np.abs(g[c] - G)) <= 1e-8 * max(1.0, np.max(np.abs(G)))
    # parameter shift on the device forward: all shifted vectors of chain 0 as one batch
    P = layers * n * 2
    shifted = np.repeat(angles[:1], 2 * P, 0)
    for p, idx in enumerate(np.ndindex(layers, n, 2)):
        shifted[2 * p][idx] += math.pi / 2
        shifted[2 * p + 1][idx] -= math.pi / 2
    ps_model = HEAEnergy(n, layers, 2 * P, chi_max=16, cutoff=1e-12)
    es = ps_model.forward(shifted).cpu().numpy()
    ps = 0.5 * (es[0::2] - es[1::2])
    adj = g[0].reshape(-1)
    assert np.max(np.abs(adj - ps)) <= 1e-5 * np.max(np.abs(ps))


def test_hea_gradient_with_truncation_matches_device_central_differences():
    from fpga_mps_simulator_b200.adjoint import HEAEnergy
    n, layers, chi = 10, 3, 4
    rng = np.random.default_rng(22)
    angles = rng.uniform(0, 2 * np.pi, (1, layers, n, 2))
    model = HEAEnergy(n, layers, 1, chi_max=chi, cutoff=1e-12)
    _, g = model.energy_and_grad(angles)
    g = g.cpu().numpy()[0]
    picks = [(0, 1, 0), (1, 4, 1), (2, 6, 0), (0, 9, 1), (2, 3, 1), (1, 7, 0)]
    h = 1e-4
    fd_model = HEAEnergy(n, layers, 2 * len(picks), chi_max=chi, cutoff=1e-12)
    shifted = np.repeat(angles, 2 * len(picks), 0)
    for p, idx in enumerate(picks):
        shifted[2 * p][idx] += h
        shifted[2 * p + 1][idx] -= h
    es = fd_model.forward(shifted).cpu().numpy()
    fd = (es[0::2] - es[1::2]) / (2 * h)
    for p, idx in enumerate(picks):
        assert abs(fd[p] - g[idx]) <= 1e-5 * max(1.0, abs(fd[p])), (idx, fd[p], g[idx])


def test_checkpointed_equals_taped_and_autograd_function():
    from fpga_mps_simulator_b200.adjoint import HEAEnergy, HEAEnergyFunction
    n, layers, nvec = 12, 3, 4
    rng = np.random.default_rng(23)
    angles = rng.uniform(0, 2 * np.pi, (nvec, layers, n, 2))
    a = HEAEnergy(n, layers, nvec, chi_max=8, checkpoint=True)
    b = HEAEnergy(n, layers, nvec, chi_max=8, checkpoint=False)
    w = torch.tensor([1.0, 0.5, -2.0, 0.0], dtype=torch.float64, device="cuda")
    ea = a.forward(angles)
    ga = a.backward(angles, w)
    eb = b.forward(angles)
    gb = b.backward(angles, w)
    assert torch.equal(ea, eb) and torch.equal(ga, gb)
    t = torch.tensor(angles, dtype=torch.float64, device="cuda", requires_grad=True)
    E = HEAEnergyFunction.apply(t, a)
    (E * w).sum().backward()
    assert torch.equal(E.detach(), ea)
    assert torch.equal(t.grad, ga)


def test_mixed_form_gradient_close_to_fp64():
    from fpga_mps_simulator_b200.adjoint import HEAEnergy
    n, layers, nvec = 16, 4, 2
    rng = np.random.default_rng(24)
    angles = rng.uniform(0, 2 * np.pi, (nvec, layers, n, 2))
    e64, g64 = HEAEnergy(n, layers, nvec, chi_max=16).energy_and_grad(angles)
    emx, gmx = HEAEnergy(n, layers, nvec, chi_max=16, precision="mixed").energy_and_grad(angles)
    assert torch.max(torch.abs(emx - e64)) < 1e-6
    assert torch.max(torch.abs(gmx - g64)) <= 1e-5 * torch.max(torch.abs(g64))


def test_xxz_initial_state_gradient_matches_central_differences():
    from fpga_mps_simulator_b200.adjoint import XXZInitialStateGradient
    from fpga_mps_simulator_b200.circuits import random_product_angles
    n, steps = 14, 3
    angles = random_product_angles(n, 31)
    model = XXZInitialStateGradient(n, steps, chi_max=16, cutoff=1e-10)
    e, g = model.energy_and_grad(angles)
    g = g.cpu().numpy()
    h = 1e-5
    for idx in [(0, 0), (3, 1), (7, 0), (13, 1), (10, 0)]:
        a = angles.copy(); a[idx] += h
        b = angles.copy(); b[idx] -= h
        fd = (model.energy(a) - model.energy(b)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, g[idx])
    assert abs(model.energy(angles) - e) < 1e-12
