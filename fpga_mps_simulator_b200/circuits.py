"""Seeded synthetic workloads for the two-site update.

All inputs are generated on the host and shared verbatim by the GPU path, the
CPU oracle and the benchmark, so every implementation sees the same gates.

* ``haar_4x4`` -- Haar-random U(4): QR of a complex Ginibre matrix
  Z = (N + iN)/sqrt(2), with the phases of diag(R) folded into Q (Mezzadri's
  construction).  The real part is drawn before the imaginary part.
* ``brickwall`` -- layers alternate even pairs (0,1),(2,3),... and odd pairs
  (1,2),(3,4),...; gates drawn in layer -> pair order.
* ``hea_layers`` -- hardware-efficient ansatz: RY(theta), RZ(phi) on every
  site, then CZ on brick-wall pairs.
* ``xxz_trotter`` -- second-order Trotter steps of the open XXZ chain with
  exact exp(-i dt h_ij) bond gates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

from .gates import gate_1q, GATE_MATRICES

__all__ = ["haar_4x4", "brickwall", "brickwall_layers", "Layer", "hea_angles",
           "hea_layers", "xxz_bond_gate", "xxz_trotter_layers",
           "random_product_angles", "CircuitSpec", "random_circuit_batch"]


def haar_4x4(rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r)
    return (q * (d / np.abs(d))[None, :]).astype(np.complex128)


@dataclass
class Layer:
    """One layer of disjoint adjacent pairs: ``sites[k]`` is the left site of pair k."""
    sites: np.ndarray                      # int32 (P,)
    gates: np.ndarray                      # complex128 (P, 4, 4)


def brickwall_layers(n: int, depth: int, seed: int) -> List[Layer]:
    rng = np.random.default_rng(seed)
    out = []
    for layer in range(depth):
        left = np.arange(layer % 2, n - 1, 2, dtype=np.int32)
        g = np.stack([haar_4x4(rng) for _ in left]) if len(left) else np.zeros((0, 4, 4), np.complex128)
        out.append(Layer(left, g))
    return out


def brickwall(n: int, depth: int, seed: int) -> List[Tuple[int, np.ndarray]]:
    """Flat (left_site, gate) list of a Haar brick-wall circuit."""
    return [(int(i), g) for L in brickwall_layers(n, depth, seed) for i, g in zip(L.sites, L.gates)]


def hea_angles(n: int, layers: int, batch: int, seed: int) -> np.ndarray:
    """Angles (batch, layers, n, 2) uniform in [0, 2*pi): [..., 0] = RY, [..., 1] = RZ."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0 * math.pi, size=(batch, layers, n, 2))


def hea_layers(n: int, angles: np.ndarray):
    """Expand one parameter vector (layers, n, 2) into (1q gates, CZ layers).

    Returns a list with one entry per ansatz layer: (g1 (n,2,2), Layer_even, Layer_odd)
    where g1[i] = RZ(phi) @ RY(theta) is the fused single-site gate.
    """
    out = []
    cz = GATE_MATRICES["cz"]
    for l in range(angles.shape[0]):
        g1 = np.stack([gate_1q("rz", [angles[l, i, 1]]) @ gate_1q("ry", [angles[l, i, 0]])
                       for i in range(n)])
        ev = np.arange(0, n - 1, 2, dtype=np.int32)
        od = np.arange(1, n - 1, 2, dtype=np.int32)
        out.append((g1, Layer(ev, np.repeat(cz[None], len(ev), 0)),
                    Layer(od, np.repeat(cz[None], len(od), 0))))
    return out


def xxz_bond_gate(dt: float, jxy: float = 1.0, jz: float = 0.5) -> np.ndarray:
    """exp(-i dt h) with h = Jxy (XX + YY) + Jz ZZ, computed from the eigenbasis."""
    x, y, z = GATE_MATRICES["x"], GATE_MATRICES["y"], GATE_MATRICES["z"]
    h = jxy * (np.kron(x, x) + np.kron(y, y)) + jz * np.kron(z, z)
    w, v = np.linalg.eigh(h)
    return (v * np.exp(-1j * dt * w)[None, :]) @ v.conj().T


def xxz_trotter_layers(n: int, steps: int, dt: float, jxy: float = 1.0, jz: float = 0.5) -> List[Layer]:
    """Second-order Trotter: half step on odd bonds, full step on even bonds, half step on odd bonds."""
    half = xxz_bond_gate(0.5 * dt, jxy, jz)
    full = xxz_bond_gate(dt, jxy, jz)
    ev = np.arange(0, n - 1, 2, dtype=np.int32)
    od = np.arange(1, n - 1, 2, dtype=np.int32)
    out = []
    for _ in range(steps):
        out.append(Layer(od, np.repeat(half[None], len(od), 0)))
        out.append(Layer(ev, np.repeat(full[None], len(ev), 0)))
        out.append(Layer(od, np.repeat(half[None], len(od), 0)))
    return out


def random_product_angles(n: int, seed: int) -> np.ndarray:
    """(n, 2) Bloch angles: theta = arccos(U[-1, 1]) (uniform on the sphere), phi ~ U[0, 2pi)."""
    rng = np.random.default_rng(seed)
    theta = np.arccos(rng.uniform(-1.0, 1.0, size=n))
    phi = rng.uniform(0.0, 2.0 * math.pi, size=n)
    return np.stack([theta, phi], axis=1)


@dataclass
class CircuitSpec:
    n: int
    depth: int
    chi_max: int
    layers: List[Layer] = field(default_factory=list)


def random_circuit_batch(count: int, seed: int, n_range=(20, 200), depth_range=(10, 40),
                         chis: Sequence[int] = (16, 32, 64)) -> List[CircuitSpec]:
    """Independent Haar brick-wall circuits of uneven size (sizes drawn first, then each circuit's gates)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_range[0], n_range[1] + 1, size=count)
    ds = rng.integers(depth_range[0], depth_range[1] + 1, size=count)
    cs = rng.choice(np.asarray(chis), size=count)
    return [CircuitSpec(int(ns[k]), int(ds[k]), int(cs[k]),
                        brickwall_layers(int(ns[k]), int(ds[k]), seed * 100003 + k))
            for k in range(count)]
