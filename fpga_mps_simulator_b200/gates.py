"""Gate matrices for the MPS two-site update (host side, complex128).

The basis convention is the one the reference MPS engine uses: a 2x2 gate acts
as ``A'[l, s', r] = sum_s G[s', s] A[l, s, r]`` and a 4x4 gate is indexed by the
combined physical index ``2*s_i + s_j`` of the adjacent pair (i, i+1), i.e.
rows/columns ordered |00>, |01>, |10>, |11> with site i as the high bit
(reference ``mps_core.py:24-43`` for the fixed table, ``:46-77`` for the
parametrised 1-qubit gates, ``:80-144`` for the parametrised 2-qubit gates).

The values are physics, not code: every entry below is written from the
textbook definition of the gate (Qiskit's conventions, which the reference
follows), and the parity tests compare each one against the reference table.
"""
from __future__ import annotations

import cmath
import math
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

__all__ = [
    "GATE_MATRICES", "gate_1q", "gate_2q", "SINGLE_QUBIT_GATES",
    "TWO_QUBIT_GATES", "swap_route", "permute_2q",
]

_R2 = 1.0 / math.sqrt(2.0)


def _m(rows) -> np.ndarray:
    return np.array(rows, dtype=np.complex128)


def _controlled(u: np.ndarray) -> np.ndarray:
    """|0><0| (x) I + |1><1| (x) u with the control on the high bit."""
    out = np.eye(4, dtype=np.complex128)
    out[2:, 2:] = u
    return out


_PAULI_X = _m([[0, 1], [1, 0]])
_PAULI_Y = _m([[0, -1j], [1j, 0]])
_PAULI_Z = _m([[1, 0], [0, -1]])
_SX = _m([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]])
_HAD = _m([[_R2, _R2], [_R2, -_R2]])

# Fixed (parameter-free) gates; reference table at mps_core.py:24-43.
GATE_MATRICES: Dict[str, np.ndarray] = {
    "id": np.eye(2, dtype=np.complex128),
    "h": _HAD,
    "x": _PAULI_X,
    "y": _PAULI_Y,
    "z": _PAULI_Z,
    "s": _m([[1, 0], [0, 1j]]),
    "sdg": _m([[1, 0], [0, -1j]]),
    "t": _m([[1, 0], [0, cmath.exp(0.25j * math.pi)]]),
    "tdg": _m([[1, 0], [0, cmath.exp(-0.25j * math.pi)]]),
    "sx": _SX,
    "sxdg": _SX.conj(),
    "cx": _controlled(_PAULI_X),
    "cz": _controlled(_PAULI_Z),
    "cy": _controlled(_PAULI_Y),
    "swap": _m([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]]),
    "iswap": _m([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]]),
    "dcx": _m([[1, 0, 0, 0], [0, 0, 0, 1], [0, 1, 0, 0], [0, 0, 1, 0]]),
}

# Name sets used by the circuit lowering (reference mps_core.py:501-510).
SINGLE_QUBIT_GATES = frozenset({
    "id", "h", "x", "y", "z", "s", "sdg", "t", "tdg", "sx", "sxdg",
    "rx", "ry", "rz", "p", "phase", "u1", "u2", "u3", "u",
})
TWO_QUBIT_GATES = frozenset({
    "cx", "cnot", "cy", "cz", "ch", "cp", "cphase", "crx", "cry", "crz",
    "csx", "swap", "iswap", "dcx", "ecr", "rxx", "ryy", "rzz",
})


def _rot(theta: float, kind: str) -> np.ndarray:
    c, s = math.cos(0.5 * theta), math.sin(0.5 * theta)
    if kind == "x":
        return _m([[c, -1j * s], [-1j * s, c]])
    if kind == "y":
        return _m([[c, -s], [s, c]])
    ph = cmath.exp(0.5j * theta)
    return _m([[ph.conjugate(), 0], [0, ph]])


def _u3(theta: float, phi: float, lam: float) -> np.ndarray:
    c, s = math.cos(0.5 * theta), math.sin(0.5 * theta)
    return _m([[c, -cmath.exp(1j * lam) * s],
               [cmath.exp(1j * phi) * s, cmath.exp(1j * (phi + lam)) * c]])


def gate_1q(name: str, params: Optional[Sequence[float]] = None) -> np.ndarray:
    """2x2 complex128 matrix of a named 1-qubit gate (reference mps_core.py:46-77)."""
    key = name.lower()
    if key in GATE_MATRICES and GATE_MATRICES[key].shape == (2, 2):
        return GATE_MATRICES[key]
    p = [float(v) for v in (params or [])]
    if key in ("rx", "ry", "rz"):
        return _rot(p[0], key[1])
    if key in ("p", "phase", "u1"):
        return _m([[1, 0], [0, cmath.exp(1j * p[0])]])
    if key == "u2":
        return _R2 * _m([[1, -cmath.exp(1j * p[1])],
                         [cmath.exp(1j * p[0]), cmath.exp(1j * (p[0] + p[1]))]])
    if key in ("u3", "u"):
        return _u3(p[0], p[1], p[2])
    raise ValueError(f"Unknown 1q gate: {name}")


def gate_2q(name: str, params: Optional[Sequence[float]] = None) -> np.ndarray:
    """4x4 complex128 matrix of a named 2-qubit gate (reference mps_core.py:80-144)."""
    key = name.lower()
    if key == "cnot":
        key = "cx"
    if key in GATE_MATRICES and GATE_MATRICES[key].shape == (4, 4):
        return GATE_MATRICES[key]
    p = [float(v) for v in (params or [])]
    if key in ("cp", "cphase"):
        out = np.eye(4, dtype=np.complex128)
        out[3, 3] = cmath.exp(1j * p[0])
        return out
    if key == "ch":
        return _controlled(_HAD)
    if key in ("crx", "cry", "crz"):
        return _controlled(_rot(p[0], key[2]))
    if key == "csx":
        return _controlled(_SX)
    if key == "ecr":
        return _R2 * _m([[0, 0, 1, 1j], [0, 0, 1j, 1], [1, -1j, 0, 0], [-1j, 1, 0, 0]])
    if key in ("rxx", "ryy"):
        c, s = math.cos(0.5 * p[0]), math.sin(0.5 * p[0])
        corner = -1j * s if key == "rxx" else 1j * s
        return _m([[c, 0, 0, corner], [0, c, -1j * s, 0],
                   [0, -1j * s, c, 0], [corner, 0, 0, c]])
    if key == "rzz":
        ph = cmath.exp(0.5j * p[0])
        return np.diag([ph.conjugate(), ph, ph, ph.conjugate()]).astype(np.complex128)
    raise ValueError(f"Unknown 2q gate: {name}")


_REVERSE_PAIR = np.array([0, 2, 1, 3])


def permute_2q(gate: np.ndarray) -> np.ndarray:
    """Re-index a 4x4 gate given on (j, i) with j > i onto (i, j).

    Swapping the two physical indices maps basis state |ab> to |ba>, which is the
    permutation [0, 2, 1, 3] on both sides (reference mps_core.py:319-322).
    """
    g = np.asarray(gate, dtype=np.complex128).reshape(4, 4)
    return g[np.ix_(_REVERSE_PAIR, _REVERSE_PAIR)]


def swap_route(i: int, j: int, name: str, params=None):
    """Nearest-neighbour lowering of a 2-qubit gate on (i, j), |i - j| > 1.

    The far qubit is swapped down until it neighbours the near one, the gate is
    applied on (lo, lo + 1), and the swaps are undone in the opposite direction
    (reference mps_core.py:151-165).  Returns (name, [a, b], params) tuples.
    """
    lo, hi = (i, j) if i < j else (j, i)
    seq = [("swap", [k - 1, k], None) for k in range(hi, lo + 1, -1)]
    seq.append((name, [lo, lo + 1], params))
    seq.extend(("swap", [k, k + 1], None) for k in range(lo + 1, hi))
    return seq
