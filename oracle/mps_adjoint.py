"""CPU adjoint of the MPS two-site update -- TEST INFRASTRUCTURE ONLY.

The reference engine (``mps_core.py`` of nasir26/fpga-mps-simulator) has no
gradients; this module is the checker for the device adjoint.  It
differentiates exactly the forward that ``OracleMPS.apply_adjacent_2q``
restates (mps_core.py:326-350 with the keep / renormalise rule of
mps_core.py:277-300), so its results are pinned by central finite
differences and by the parameter-shift rule in ``tests/test_adjoint_oracle.py``.

Conventions.  For a real loss L and a complex array z the cotangent is
z_bar = dL/dRe(z) + i dL/dIm(z) (= 2 dL/dz*), so that
dL = Re sum(conj(z_bar) dz).  With it, y = W x gives x_bar = W^H y_bar.

Truncated SVD backward.  M = U S V^H (thin, all r = min(m, n) triplets);
the forward keeps k of them.  The cotangents of the discarded columns are
zero, and the exact derivative of the kept factors is the full thin-SVD
backward with those zeros:

    M_bar = U G V^H + (I - U U^H) U_bar S^-1 V^H + U S^-1 V_bar^H (I - V V^H)
    G_ij  = s_j F_ij (P - P^H)_ij + s_i F_ij (Q - Q^H)_ij        (i != j)
    G_ii  = S_bar_i + i (Im P_ii - Im Q_ii) / (2 s_i)
    P = U^H U_bar,  Q = V^H V_bar,
    F_ij  = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + eps)          (Lorentzian-broadened
                                                                 1/(s_j^2 - s_i^2))

with eps = (BROADEN * s_0^2)^2.  The kept/discarded coupling terms (i kept,
j discarded) are what distinguish this from the rank-k formula.  The
diagonal imaginary term fixes the U(1) gauge of each triplet symmetrically
(diag(U^H dU) = -diag(V^H dV)), which makes the formula covariant under
M -> M^H; the losses differentiated here are invariant under the bond gauge,
so any fixing gives the same gradient.

The loss side: L = <psi|H|psi> / <psi|psi> for a matrix-product operator H;
the cotangent of site k is 2 (H_eff A_k - L N_eff A_k) / <psi|psi>.  The
overall scale (norm_log, the S renormalisation) drops out of such losses.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np
import scipy.linalg as sla

__all__ = ["BROADEN", "update_forward", "svd_backward", "update_backward", "update_backward_given_outputs",
           "tfim_mpo", "nn_mpo", "mpo_energy", "mpo_energy_grad", "apply1q_backward",
           "hea_energy", "hea_energy_grad", "rot_gate", "rot_gate_derivs"]

BROADEN = 1e-12


def update_forward(A: np.ndarray, B: np.ndarray, G: np.ndarray, chi_max: int, cutoff: float):
    """One two-site update with the reference's semantics; returns (A', B', aux).

    aux holds M (the gated theta as (2 cl) x (2 cr)), the full thin SVD
    (U, S, Vh), the kept count and the kept-norm divisor.
    """
    cl, cr = A.shape[0], B.shape[2]
    theta = np.einsum("lpm,mqr->lpqr", A, B).reshape(cl, 4, cr)
    theta = np.einsum("st,ltr->lsr", np.asarray(G, np.complex128).reshape(4, 4), theta)
    M = theta.reshape(2 * cl, 2 * cr)
    U, S, Vh = sla.svd(M, full_matrices=False, lapack_driver="gesdd")
    thr = cutoff * S[0] if S.size else 0.0
    keep = int(min(max(int(np.count_nonzero(S > thr)), 1), chi_max))
    nrm = float(np.linalg.norm(S[:keep]))
    div = nrm if nrm > 1e-15 else 1.0
    sq = np.sqrt(S[:keep] / div)
    Ap = (U[:, :keep] * sq[None, :]).reshape(cl, 2, keep)
    Bp = (sq[:, None] * Vh[:keep]).reshape(keep, 2, cr)
    return Ap, Bp, {"M": M, "U": U, "S": S, "Vh": Vh, "keep": keep, "div": div}


def _broadened_inverse(S: np.ndarray) -> np.ndarray:
    d = S[None, :] ** 2 - S[:, None] ** 2          # d_ij = s_j^2 - s_i^2
    eps = (BROADEN * (S[0] ** 2 if S.size else 1.0)) ** 2
    F = d / (d * d + eps)
    np.fill_diagonal(F, 0.0)
    return F


def svd_backward(U: np.ndarray, S: np.ndarray, V: np.ndarray, Ubar: np.ndarray, Vbar: np.ndarray,
                 Sbar: np.ndarray) -> np.ndarray:
    """M_bar for M = U diag(S) V^H given cotangents of the first k columns.

    U (m, r), S (r,), V (n, r) are the full thin factors; Ubar (m, k),
    Vbar (n, k), Sbar (k,) the cotangents of the kept triplets.
    """
    r, k = S.size, Ubar.shape[1]
    Ub = np.zeros((U.shape[0], r), np.complex128)
    Vb = np.zeros((V.shape[0], r), np.complex128)
    Ub[:, :k], Vb[:, :k] = Ubar, Vbar
    Sb = np.zeros(r)
    Sb[:k] = Sbar
    P = U.conj().T @ Ub
    Q = V.conj().T @ Vb
    F = _broadened_inverse(S)
    G = (F * (P - P.conj().T)) * S[None, :] + S[:, None] * (F * (Q - Q.conj().T))
    inv = np.zeros(r)
    inv[:k] = 1.0 / S[:k]
    G = G + np.diag(Sb + 0.5j * (np.imag(np.diag(P)) - np.imag(np.diag(Q))) * inv)
    Mbar = U @ G @ V.conj().T
    Mbar += (Ub - U @ P) * inv[None, :] @ V.conj().T
    Mbar += U @ (inv[:, None] * (Vb.conj().T - Q.conj().T @ V.conj().T))
    return Mbar


def _theta_backward(A, B, G, Mbar, need_gate: bool):
    cl, cm, cr = A.shape[0], A.shape[2], B.shape[2]
    tpbar = Mbar.reshape(cl, 4, cr)                      # cotangent of the gated theta
    Gm = np.asarray(G, np.complex128).reshape(4, 4)
    tbar = np.einsum("ts,ltr->lsr", Gm.conj(), tpbar)     # G^H applied
    Gbar = None
    if need_gate:
        theta = np.einsum("lpm,mqr->lpqr", A, B).reshape(cl, 4, cr)
        Gbar = np.einsum("ltr,lsr->ts", tpbar, theta.conj())
    tb = tbar.reshape(2 * cl, 2 * cr)
    Abar = (tb @ B.reshape(cm, 2 * cr).conj().T).reshape(cl, 2, cm)
    Bbar = (A.reshape(2 * cl, cm).conj().T @ tb).reshape(cm, 2, cr)
    return Abar, Bbar, Gbar


def update_backward(A, B, G, aux, Apbar, Bpbar, need_gate: bool = False):
    """(A_bar, B_bar[, G_bar]) of one update from the cotangents of (A', B')."""
    k, div = aux["keep"], aux["div"]
    U, S, V = aux["U"], aux["S"], aux["Vh"].conj().T
    s = S[:k] / div
    sq = np.sqrt(s)
    Pa = Apbar.reshape(-1, k)
    Pb = Bpbar.reshape(k, -1)
    Ubar = Pa * sq[None, :]
    Vbar = (sq[:, None] * Pb).conj().T
    sbar = (np.real(np.sum(Pa.conj() * U[:, :k], 0)) + np.real(np.sum(Pb.conj() * aux["Vh"][:k], 1))) / (2 * sq)
    Sbar = (sbar - s * np.dot(s, sbar)) / div
    Mbar = svd_backward(U, S, V, Ubar, Vbar, Sbar)
    return _theta_backward(A, B, G, Mbar, need_gate)


def update_backward_given_outputs(A, B, G, Ap, Bp, Apbar, Bpbar, need_gate: bool = False):
    """The same backward with the kept factors taken from given outputs (A', B').

    The SVD gauge of the kept triplets is the one the outputs carry (any
    implementation's forward); the discarded triplets come from this
    module's own SVD of M (their gauge does not enter the result).
    """
    cl, cr = A.shape[0], B.shape[2]
    k = Ap.shape[2]
    theta = np.einsum("lpm,mqr->lpqr", A, B).reshape(cl, 4, cr)
    M = np.einsum("st,ltr->lsr", np.asarray(G, np.complex128).reshape(4, 4), theta).reshape(2 * cl, 2 * cr)
    U0, S, Vh0 = sla.svd(M, full_matrices=False, lapack_driver="gesdd")
    a = Ap.reshape(2 * cl, k)
    b = Bp.reshape(k, 2 * cr)
    s = np.real(np.sum(a.conj() * a, 0))
    nrm = float(np.linalg.norm(S[:k]))
    div = nrm if nrm > 1e-15 else 1.0
    U = U0.copy()
    Vh = Vh0.copy()
    U[:, :k] = a / np.sqrt(s)[None, :]
    Vh[:k] = b / np.sqrt(s)[:, None]
    S = S.copy()
    S[:k] = s * div
    aux = {"M": M, "U": U, "S": S, "Vh": Vh, "keep": k, "div": div}
    return update_backward(A, B, G, aux, Apbar, Bpbar, need_gate)


# -- matrix-product operators -------------------------------------------------
_I2 = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], np.complex128)
_Y = np.array([[0, -1j], [1j, 0]], np.complex128)
_Z = np.array([[1, 0], [0, -1]], np.complex128)


def nn_mpo(n: int, onsite: Sequence[np.ndarray], bond: Sequence[Tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    """MPO of H = sum_i onsite[i] + sum_i sum_p (O_p on i)(P_p on i+1), as (n, D, D, 2, 2).

    D = 2 + len(bond).  Index D-1 is the "nothing placed yet" state (the left
    boundary), index 0 the "complete" state (the right boundary); W[a, b]
    moves from state a (left bond) to state b (right bond).
    """
    nb = len(bond)
    D = 2 + nb
    W = np.zeros((n, D, D, 2, 2), np.complex128)
    for k in range(n):
        W[k, 0, 0] = _I2
        W[k, D - 1, D - 1] = _I2
        W[k, D - 1, 0] = onsite[k]
        for p, (o, q) in enumerate(bond):
            W[k, D - 1, 1 + p] = o
            W[k, 1 + p, 0] = q
    return W


def tfim_mpo(n: int, J: float = 1.0, h: float = 1.0) -> np.ndarray:
    """H = -J sum Z_i Z_{i+1} - h sum X_i."""
    return nn_mpo(n, [-h * _X] * n, [(-J * _Z, _Z)])


def _envs(sites, W):
    """Left and right MPO environments; L[k] is (D, chi, chi) before site k (bra index first)."""
    n, D = len(sites), W.shape[1]
    L = [None] * (n + 1)
    R = [None] * (n + 1)
    L[0] = np.zeros((D, 1, 1), np.complex128)
    L[0][D - 1] = 1.0
    for k in range(n):
        a = sites[k]
        t = np.einsum("axy,ytv->axtv", L[k], a)
        t = np.einsum("axtv,abst->bxsv", t, W[k])
        L[k + 1] = np.einsum("bxsv,xsu->buv", t, a.conj())
    R[n] = np.zeros((D, 1, 1), np.complex128)
    R[n][0] = 1.0
    for k in range(n - 1, -1, -1):
        a = sites[k]
        t = np.einsum("ytv,buv->ytbu", a, R[k + 1])
        t = np.einsum("ytbu,abst->ysau", t, W[k])
        R[k] = np.einsum("ysau,xsu->axy", t, a.conj())
    return L, R


def _identity_mpo(n: int) -> np.ndarray:
    W = np.zeros((n, 1, 1, 2, 2), np.complex128)
    W[:, 0, 0] = _I2
    return W


def mpo_energy(sites, W) -> Tuple[float, float]:
    """(<psi|H|psi>, <psi|psi>) of an MPS given as site tensors (norm_log excluded)."""
    L, _ = _envs(sites, W)
    Ln, _ = _envs(sites, _identity_mpo(len(sites)))
    return float(np.real(L[-1][0, 0, 0])), float(np.real(Ln[-1][0, 0, 0]))


def _heff(L, R, W, a):
    t = np.einsum("axy,ytv->axtv", L, a)
    t = np.einsum("axtv,abst->bxsv", t, W)
    return np.einsum("bxsv,buv->xsu", t, R)


def mpo_energy_grad(sites, W) -> Tuple[float, List[np.ndarray]]:
    """L = <H>/<1> and the cotangents 2 (H_eff A_k - L N_eff A_k) / <1> of every site."""
    n = len(sites)
    L, R = _envs(sites, W)
    I = _identity_mpo(n)
    Ln, Rn = _envs(sites, I)
    E = float(np.real(L[-1][0, 0, 0]))
    N = float(np.real(Ln[-1][0, 0, 0]))
    loss = E / N
    grads = []
    for k in range(n):
        he = _heff(L[k], R[k + 1], W[k], sites[k])
        ne = _heff(Ln[k], Rn[k + 1], I[k], sites[k])
        grads.append(2.0 * (he - loss * ne) / N)
    return loss, grads


def apply1q_backward(A, G, Apbar):
    """A' = G A on the physical index: (A_bar, G_bar)."""
    Abar = np.einsum("ts,ltr->lsr", np.asarray(G).conj(), Apbar)
    Gbar = np.einsum("ltr,lsr->ts", Apbar, A.conj())
    return Abar, Gbar


# -- hardware-efficient ansatz -------------------------------------------------
def rot_gate(theta: float, phi: float) -> np.ndarray:
    """RZ(phi) RY(theta) with RY = exp(-i theta Y/2), RZ = exp(-i phi Z/2)."""
    c, s = math.cos(0.5 * theta), math.sin(0.5 * theta)
    ry = np.array([[c, -s], [s, c]], np.complex128)
    rz = np.diag([np.exp(-0.5j * phi), np.exp(0.5j * phi)])
    return rz @ ry


def rot_gate_derivs(theta: float, phi: float):
    """(dG/dtheta, dG/dphi) of rot_gate."""
    g = rot_gate(theta, phi)
    c, s = math.cos(0.5 * theta), math.sin(0.5 * theta)
    ry = np.array([[c, -s], [s, c]], np.complex128)
    rz = np.diag([np.exp(-0.5j * phi), np.exp(0.5j * phi)])
    return rz @ (-0.5j * _Y @ ry), -0.5j * _Z @ g


_CZ = np.diag([1, 1, 1, -1]).astype(np.complex128)


def _hea_ops(n: int, angles: np.ndarray):
    for l in range(angles.shape[0]):
        yield ("1q", l)
        yield ("2q", list(range(0, n - 1, 2)))
        yield ("2q", list(range(1, n - 1, 2)))


def _product_zero(n):
    out = []
    for _ in range(n):
        t = np.zeros((1, 2, 1), np.complex128)
        t[0, 0, 0] = 1.0
        out.append(t)
    return out


def hea_energy(angles: np.ndarray, W: np.ndarray, chi_max: int, cutoff: float) -> float:
    """Normalised <H> after the ansatz (RY, RZ on every site, CZ on even then odd pairs, per layer)."""
    n = angles.shape[1]
    sites = _product_zero(n)
    for op, arg in _hea_ops(n, angles):
        if op == "1q":
            for i in range(n):
                g = rot_gate(angles[arg, i, 0], angles[arg, i, 1])
                sites[i] = np.einsum("ts,lsr->ltr", g, sites[i])
        else:
            for i in arg:
                sites[i], sites[i + 1], _ = update_forward(sites[i], sites[i + 1], _CZ, chi_max, cutoff)
    E, N = mpo_energy(sites, W)
    return E / N


def hea_energy_grad(angles: np.ndarray, W: np.ndarray, chi_max: int, cutoff: float):
    """(loss, dloss/dangles) by the hand-written adjoint (tape kept in memory)."""
    n = angles.shape[1]
    sites = _product_zero(n)
    tape = []
    for op, arg in _hea_ops(n, angles):
        if op == "1q":
            pre = [t.copy() for t in sites]
            for i in range(n):
                g = rot_gate(angles[arg, i, 0], angles[arg, i, 1])
                sites[i] = np.einsum("ts,lsr->ltr", g, sites[i])
            tape.append(("1q", arg, pre))
        else:
            recs = []
            for i in arg:
                A, B = sites[i], sites[i + 1]
                sites[i], sites[i + 1], aux = update_forward(A, B, _CZ, chi_max, cutoff)
                recs.append((i, A, B, aux))
            tape.append(("2q", arg, recs))
    loss, cot = mpo_energy_grad(sites, W)
    grad = np.zeros_like(angles)
    for op, arg, rec in reversed(tape):
        if op == "1q":
            for i in range(n):
                th, ph = angles[arg, i]
                g = rot_gate(th, ph)
                cot[i], gbar = apply1q_backward(rec[i], g, cot[i])
                dth, dph = rot_gate_derivs(th, ph)
                grad[arg, i, 0] = np.real(np.sum(gbar.conj() * dth))
                grad[arg, i, 1] = np.real(np.sum(gbar.conj() * dph))
        else:
            for i, A, B, aux in reversed(rec):
                cot[i], cot[i + 1], _ = update_backward(A, B, _CZ, aux, cot[i], cot[i + 1])
    return loss, grad
