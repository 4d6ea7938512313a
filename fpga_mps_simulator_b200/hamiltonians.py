"""Nearest-neighbour Hamiltonians as matrix-product operators.

Layout (what ``mpsb_mpo_energy_grad`` reads): ``W`` of shape (n, D, D, 2, 2)
complex128, ``W[k, a, b]`` the operator that moves the automaton from state a
(left bond) to state b (right bond) at site k, acting as |s><t| at [s, t].
State D-1 is "nothing placed yet" (left boundary), state 0 "complete" (right
boundary); ``W[k, D-1, D-1] = W[k, 0, 0] = I``.  For
H = sum_k h_k + sum_k sum_p O_p(k) P_p(k+1) the bond is D = 2 + #products.
"""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

__all__ = ["nn_mpo", "tfim_mpo", "zz_mpo", "check_mpo"]

_I2 = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], np.complex128)
_Z = np.array([[1, 0], [0, -1]], np.complex128)


def nn_mpo(n: int, onsite: Sequence[np.ndarray], bond: Sequence[Tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    """MPO of sum_k onsite[k] + sum_k sum_p bond[p][0] (site k) bond[p][1] (site k+1)."""
    nb = len(bond)
    D = 2 + nb
    W = np.zeros((n, D, D, 2, 2), np.complex128)
    for k in range(n):
        W[k, 0, 0] = _I2
        W[k, D - 1, D - 1] = _I2
        W[k, D - 1, 0] = np.asarray(onsite[k], np.complex128)
        for p, (o, q) in enumerate(bond):
            W[k, D - 1, 1 + p] = np.asarray(o, np.complex128)
            W[k, 1 + p, 0] = np.asarray(q, np.complex128)
    return W


def tfim_mpo(n: int, J: float = 1.0, h: float = 1.0) -> np.ndarray:
    """Transverse-field Ising H = -J sum Z_i Z_{i+1} - h sum X_i (open chain)."""
    return nn_mpo(n, [-h * _X] * n, [(-J * _Z, _Z)])


def zz_mpo(n: int) -> np.ndarray:
    """sum_i Z_i Z_{i+1} (open chain)."""
    return nn_mpo(n, [np.zeros((2, 2), np.complex128)] * n, [(_Z, _Z)])


def check_mpo(W: np.ndarray, n: int) -> np.ndarray:
    """Validate the lower-triangular boundary convention the device kernels rely on."""
    W = np.ascontiguousarray(np.asarray(W, np.complex128))
    if W.ndim != 5 or W.shape[0] != n or W.shape[1] != W.shape[2] or W.shape[3:] != (2, 2):
        raise ValueError(f"MPO must have shape (n={n}, D, D, 2, 2), got {W.shape}")
    D = W.shape[1]
    if not (1 <= D <= 16):
        raise ValueError("MPO bond must be in [1, 16]")
    for k in range(n):
        if not (np.allclose(W[k, 0, 0], _I2) and np.allclose(W[k, D - 1, D - 1], _I2)):
            raise ValueError("W[k, 0, 0] and W[k, D-1, D-1] must be the identity")
        if D > 1 and (np.any(W[k, 0, 1:] != 0) or np.any(W[k, :D - 1, D - 1] != 0)):
            raise ValueError("no transition may leave state 0 or enter state D-1")
    return W
