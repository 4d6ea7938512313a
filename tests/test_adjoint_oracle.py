"""The CPU adjoint (oracle/mps_adjoint.py) pinned by central finite
differences and by the parameter-shift rule -- no GPU.  These pins are what
make it a valid checker for the device adjoint."""
import math

import numpy as np
import pytest

from oracle.mps_adjoint import (hea_energy, hea_energy_grad, mpo_energy, mpo_energy_grad, tfim_mpo,
                                update_backward, update_backward_given_outputs, update_forward)


def _rand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _haar(rng):
    q, r = np.linalg.qr(_rand(rng, (4, 4)))
    return q * (np.diag(r) / np.abs(np.diag(r)))[None, :]


def _chain_loss(sites, i, G, chi, cut, W):
    s = list(sites)
    s[i], s[i + 1], _ = update_forward(s[i], s[i + 1], G, chi, cut)
    E, N = mpo_energy(s, W)
    return E / N


@pytest.mark.parametrize("chi,bonds", [(64, (1, 2, 4, 2, 1)), (3, (1, 2, 4, 2, 1)), (2, (1, 2, 3, 2, 1))])
def test_update_backward_matches_central_differences(chi, bonds):
    rng = np.random.default_rng(chi * 7 + bonds[2])
    n = len(bonds) - 1
    sites = [_rand(rng, (bonds[k], 2, bonds[k + 1])) for k in range(n)]
    G = _haar(rng) + 0.3 * _rand(rng, (4, 4))     # non-unitary: the gate cotangent is general
    W = tfim_mpo(n, 1.0, 0.7)
    i = 1
    A, B = sites[i], sites[i + 1]
    Ap, Bp, aux = update_forward(A, B, G, chi, 1e-12)
    s2 = list(sites)
    s2[i], s2[i + 1] = Ap, Bp
    loss, cot = mpo_energy_grad(s2, W)
    Abar, Bbar, Gbar = update_backward(A, B, G, aux, cot[i], cot[i + 1], need_gate=True)
    h = 1e-6
    for which, X, Xbar in (("A", A, Abar), ("B", B, Bbar), ("G", G, Gbar)):
        for idx in list(np.ndindex(X.shape))[:12]:
            for unit in (1.0, 1j):
                def f(t):
                    Xp = X.copy()
                    Xp[idx] += t * unit
                    s = list(sites)
                    a, b, g = A, B, G
                    if which == "A":
                        s[i] = Xp
                    elif which == "B":
                        s[i + 1] = Xp
                    else:
                        g = Xp
                    return _chain_loss(s, i, g, chi, 1e-12, W)
                fd = (f(h) - f(-h)) / (2 * h)
                an = np.real(np.conj(Xbar[idx]) * unit)
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (which, idx, unit, fd, an)


def test_backward_from_given_outputs_equals_backward_from_aux():
    rng = np.random.default_rng(3)
    A, B = _rand(rng, (3, 2, 4)), _rand(rng, (4, 2, 2))
    G = _haar(rng)
    Ap, Bp, aux = update_forward(A, B, G, 3, 1e-12)
    # another gauge of the same factorisation: per-triplet phases
    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, Ap.shape[2]))
    Ap2, Bp2 = Ap * ph[None, None, :], Bp * ph.conj()[:, None, None]
    Cbar_a, Cbar_b = _rand(rng, Ap.shape), _rand(rng, Bp.shape)
    r1 = update_backward(A, B, G, aux, Cbar_a, Cbar_b)
    r2 = update_backward_given_outputs(A, B, G, Ap, Bp, Cbar_a, Cbar_b)
    for x, y in zip(r1[:2], r2[:2]):
        np.testing.assert_allclose(x, y, atol=1e-11)
    # cotangents carried into the other gauge give the same (gauge-invariant) result
    r3 = update_backward_given_outputs(A, B, G, Ap2, Bp2, Cbar_a * ph[None, None, :], Cbar_b * ph.conj()[:, None, None])
    for x, y in zip(r1[:2], r3[:2]):
        np.testing.assert_allclose(x, y, atol=1e-11)


def test_mpo_energy_matches_dense_tfim():
    rng = np.random.default_rng(5)
    n = 5
    sites = [_rand(rng, (1 if k == 0 else 2, 2, 1 if k == n - 1 else 2)) for k in range(n)]
    E, N = mpo_energy(sites, tfim_mpo(n, 1.0, 1.0))
    psi = sites[0][0]
    for k in range(1, n):
        psi = np.einsum("xc,csd->xsd", psi, sites[k]).reshape(-1, sites[k].shape[2])
    psi = psi[:, 0]
    X = np.array([[0, 1], [1, 0]]); Z = np.diag([1, -1]); I = np.eye(2)

    def op(ops):
        m = np.array([[1.0]])
        for k in range(n):
            m = np.kron(m, ops.get(k, I))
        return m
    H = sum(-op({k: Z, k + 1: Z}) for k in range(n - 1)) + sum(-op({k: X}) for k in range(n))
    assert abs(E - np.vdot(psi, H @ psi).real) < 1e-10
    assert abs(N - np.vdot(psi, psi).real) < 1e-10


def _param_shift(angles, W, chi, cut):
    g = np.zeros_like(angles)
    for idx in np.ndindex(angles.shape):
        a = angles.copy(); a[idx] += math.pi / 2
        b = angles.copy(); b[idx] -= math.pi / 2
        g[idx] = 0.5 * (hea_energy(a, W, chi, cut) - hea_energy(b, W, chi, cut))
    return g


def test_hea_adjoint_matches_parameter_shift_and_fd():
    n, layers = 6, 2
    rng = np.random.default_rng(11)
    angles = rng.uniform(0, 2 * np.pi, (layers, n, 2))
    W = tfim_mpo(n)
    loss, grad = hea_energy_grad(angles, W, 64, 1e-12)
    assert abs(loss - hea_energy(angles, W, 64, 1e-12)) < 1e-12
    ps = _param_shift(angles, W, 64, 1e-12)
    assert np.max(np.abs(grad - ps)) <= 1e-5 * np.max(np.abs(ps))
    h = 1e-4
    for idx in [(0, 0, 0), (0, 3, 1), (1, 5, 0), (1, 2, 1)]:
        a = angles.copy(); a[idx] += h
        b = angles.copy(); b[idx] -= h
        fd = (hea_energy(a, W, 64, 1e-12) - hea_energy(b, W, 64, 1e-12)) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd))


def test_hea_adjoint_with_truncation_matches_fd():
    n, layers, chi = 8, 3, 3
    rng = np.random.default_rng(12)
    angles = rng.uniform(0, 2 * np.pi, (layers, n, 2))
    W = tfim_mpo(n)
    loss, grad = hea_energy_grad(angles, W, chi, 1e-12)
    h = 1e-5
    for idx in [(0, 1, 0), (1, 4, 1), (2, 6, 0), (0, 7, 1), (2, 3, 1)]:
        a = angles.copy(); a[idx] += h
        b = angles.copy(); b[idx] -= h
        fd = (hea_energy(a, W, chi, 1e-12) - hea_energy(b, W, chi, 1e-12)) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, grad[idx])
