"""CPU oracle for the MPS two-site update -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy/scipy, the algorithm of the reference engine
``mps_core.py`` (nasir26/fpga-mps-simulator) for the hot path: contract two
neighbouring site tensors, apply a 4x4 gate, truncated SVD (LAPACK gesdd via
``scipy.linalg.svd``), renormalise, split with sqrt(S) on both sides.  Every
method cites the reference lines it follows.

It is the checker for the CUDA path and the CPU baseline that ``bench.py``
times; nothing in the product imports it.  Its fidelity to the reference is
pinned by ``tests/test_oracle.py`` against ``tests/golden/*.npz``, which
``tests/golden/make_golden.py`` generated by running the reference module
itself.

Additions that the reference does not have (transfer-matrix expectations and
single amplitudes for chains too long for a statevector, and a dense
statevector simulator for exact comparisons) follow the conventions fixed by
the reference's ``get_statevector`` (``mps_core.py:433-461``): site 0 is the
most significant bit of the contraction order, the amplitude carries
``exp(norm_log)``, and the returned statevector is in Qiskit little-endian
order.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np
import scipy.linalg as sla

__all__ = ["OracleMPS", "dense_zero_state", "dense_apply_1q", "dense_apply_2q",
           "dense_expect_pauli", "fidelity", "haar_4x4_oracle"]

_PERM_REVERSED = np.array([0, 2, 1, 3])
_SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)


class OracleMPS:
    """Reference-semantics MPS (site tensors (chi_l, 2, chi_r), complex128).

    Mirrors ``MPSState`` at ``mps_core.py:172-201``: the chain starts in
    |0...0> with every bond of dimension 1, ``norm_log`` starts at 0.
    ``record`` keeps, per two-site update, the full singular-value spectrum,
    the kept count and the two ``norm_log`` increments, which is the
    gauge-invariant data the parity tests compare.
    """

    def __init__(self, n: int, chi_max: int = 256, svd_cutoff: float = 1e-12, record: bool = True):
        self.n = int(n)
        self.chi_max = int(chi_max)
        self.svd_cutoff = float(svd_cutoff)
        self.norm_log = 0.0
        self.record = record
        self.log: List[Dict] = []
        self.sites: List[np.ndarray] = []
        for _ in range(self.n):
            t = np.zeros((1, 2, 1), dtype=np.complex128)
            t[0, 0, 0] = 1.0
            self.sites.append(t)

    # -- bookkeeping (mps_core.py:197-217) ---------------------------------
    def copy(self) -> "OracleMPS":
        o = OracleMPS(self.n, self.chi_max, self.svd_cutoff, self.record)
        o.sites = [t.copy() for t in self.sites]
        o.norm_log = self.norm_log
        return o

    def bond_dims(self) -> List[int]:
        return [int(self.sites[k].shape[2]) for k in range(self.n - 1)]

    def max_bond(self) -> int:
        return max(self.bond_dims()) if self.n > 1 else 1

    # -- gates ---------------------------------------------------------------
    def apply_1q(self, site: int, gate: np.ndarray) -> None:
        """A'[l, s', r] = sum_s G[s', s] A[l, s, r]  (mps_core.py:267-273)."""
        self.sites[site] = np.einsum("ts,lsr->ltr", np.asarray(gate, np.complex128), self.sites[site])

    def svd_truncate(self, mat: np.ndarray):
        """Truncated SVD with the reference's exact keep / renormalise rule.

        mps_core.py:277-300: gesdd SVD; threshold = cutoff * S[0]; keep =
        clip(#(S > threshold), 1, chi_max); when truncating, add
        0.5*log(1 - dropped/max(sum S^2, 1e-300)) if dropped > 0; then divide
        the kept S by its 2-norm when that norm exceeds 1e-15, adding its log.
        """
        u, s, vh = sla.svd(mat, full_matrices=False, lapack_driver="gesdd")
        thr = self.svd_cutoff * s[0] if s.size else 0.0
        keep = int(min(max(int(np.count_nonzero(s > thr)), 1), self.chi_max))
        d1 = 0.0
        if keep < s.size:
            dropped = float(np.sum(s[keep:] ** 2))
            if dropped > 0:
                d1 = 0.5 * math.log(1.0 - dropped / max(float(np.sum(s ** 2)), 1e-300))
        self.norm_log += d1
        kept = s[:keep]
        nrm = float(np.linalg.norm(kept))
        d2 = 0.0
        if nrm > 1e-15:
            d2 = math.log(nrm)
            kept = kept / nrm
        self.norm_log += d2
        if self.record:
            self.log.append({"S": s.copy(), "keep": keep, "d_trunc": d1, "d_norm": d2})
        return u[:, :keep], np.sqrt(kept), vh[:keep, :]

    def apply_adjacent_2q(self, i: int, gate: np.ndarray) -> None:
        """contract -> gate -> truncated SVD -> sqrt(S) split (mps_core.py:326-350)."""
        a, b = self.sites[i], self.sites[i + 1]
        cl, cr = a.shape[0], b.shape[2]
        theta = np.einsum("lpm,mqr->lpqr", a, b).reshape(cl, 4, cr)
        theta = np.einsum("st,ltr->lsr", np.asarray(gate, np.complex128).reshape(4, 4), theta)
        u, sq, vh = self.svd_truncate(theta.reshape(2 * cl, 2 * cr))
        k = sq.size
        self.sites[i] = (u * sq[None, :]).reshape(cl, 2, k)
        self.sites[i + 1] = (sq[:, None] * vh).reshape(k, 2, cr)

    # the reference spells it with a leading underscore
    _apply_adjacent_2q = apply_adjacent_2q

    def apply_2q(self, i: int, j: int, gate: np.ndarray) -> None:
        """Dispatch of mps_core.py:304-324.

        Non-adjacent pairs are lowered to a SWAP chain and the gate is applied
        on (lo, lo+1) *without* re-indexing it, as the reference does; an
        adjacent pair given as (i+1, i) re-indexes the gate with [0,2,1,3].
        """
        g = np.asarray(gate, np.complex128).reshape(4, 4)
        if abs(i - j) != 1:
            lo, hi = min(i, j), max(i, j)
            for k in range(hi, lo + 1, -1):
                self.apply_2q(k - 1, k, _SWAP)
            self.apply_2q(lo, lo + 1, g)
            for k in range(lo + 1, hi):
                self.apply_2q(k, k + 1, _SWAP)
            return
        if i > j:
            i, j = j, i
            g = g[np.ix_(_PERM_REVERSED, _PERM_REVERSED)]
        self.apply_adjacent_2q(i, g)

    def reset(self, site: int) -> None:
        """Project a site on sigma=0 and renormalise it (fpga_mps_simulator.py:530-552)."""
        t = self.sites[site].copy()
        t[:, 1, :] = 0.0
        nm = float(np.linalg.norm(t))
        if nm > 1e-15:
            t /= nm
        else:
            t = np.zeros_like(t)
            t[0, 0, 0] = 1.0
        self.sites[site] = t

    # -- canonical forms (mps_core.py:219-261) ---------------------------------
    def left_normalize_site(self, i: int) -> None:
        """QR of site i as (chi_l*2) x chi_r; Q stays, R is absorbed into site i+1."""
        a = self.sites[i]
        cl, d, cr = a.shape
        q, r = np.linalg.qr(a.reshape(cl * d, cr))
        self.sites[i] = q.reshape(cl, d, q.shape[1])
        if i + 1 < self.n:
            self.sites[i + 1] = np.tensordot(r, self.sites[i + 1], axes=([1], [0]))

    def right_normalize_site(self, i: int) -> None:
        """LQ of site i as chi_l x (2*chi_r) (QR of its conjugate transpose); L absorbed into site i-1."""
        a = self.sites[i]
        cl, d, cr = a.shape
        q, r = np.linalg.qr(a.reshape(cl, d * cr).T.conj())
        lmat = r.T.conj()
        b = q.T.conj()
        self.sites[i] = b.reshape(b.shape[0], d, cr)
        if i - 1 >= 0:
            self.sites[i - 1] = np.tensordot(self.sites[i - 1], lmat, axes=([2], [0]))

    def left_canonicalize(self) -> None:
        for i in range(self.n - 1):
            self.left_normalize_site(i)

    def right_canonicalize(self) -> None:
        for i in range(self.n - 1, 0, -1):
            self.right_normalize_site(i)

    def entanglement_entropy(self, bond: int) -> float:
        """mps_core.py:465-483: SVD of the contracted left block (sites 0..bond), S > 1e-15."""
        if bond < 0 or bond >= self.n - 1:
            raise ValueError(f"bond {bond} out of range [0, {self.n - 2}]")
        a = self.sites[0][0, :, :]
        for i in range(1, bond + 1):
            a = np.tensordot(a, self.sites[i], axes=([1], [0])).reshape(-1, self.sites[i].shape[2])
        s = sla.svd(a, full_matrices=False, compute_uv=False)
        s = s[s > 1e-15]
        p = s ** 2
        p = p / p.sum()
        return -float(np.sum(p * np.log(np.maximum(p, 1e-300))))

    def bond_spectrum(self, bond: int) -> np.ndarray:
        """mps_core.py:485-494: left-normalise sites 0..bond of a copy, SVD of site `bond`."""
        m = self.copy()
        for i in range(bond + 1):
            m.left_normalize_site(i)
        a = m.sites[bond]
        return sla.svd(a.reshape(-1, a.shape[2]), full_matrices=False, compute_uv=False)

    # -- read-out -------------------------------------------------------------
    def statevector(self) -> np.ndarray:
        """Dense amplitudes in Qiskit order, including exp(norm_log) (mps_core.py:433-461)."""
        if self.n > 24:
            raise ValueError("statevector limited to n <= 24")
        psi = self.sites[0][0]                         # (2, chi)
        for k in range(1, self.n):
            psi = np.einsum("xc,csd->xsd", psi, self.sites[k]).reshape(-1, self.sites[k].shape[2])
        psi = psi[:, 0].copy()
        if self.norm_log != 0.0:
            psi *= math.exp(self.norm_log)
        return psi.reshape([2] * self.n).transpose(list(range(self.n - 1, -1, -1))).reshape(-1)

    get_statevector = statevector

    def amplitude(self, bits: Sequence[int]) -> complex:
        """<b_0 ... b_{n-1}|psi> with b_k the value of qubit k, including exp(norm_log)."""
        v = np.ones((1,), dtype=np.complex128)
        for k in range(self.n):
            v = v @ self.sites[k][:, int(bits[k]), :]
        return complex(v[0] * math.exp(self.norm_log))

    def _transfer_left(self):
        """Left environments E_k (E_0 = [[1]]), each trace-normalised, with the log scales."""
        envs, logs = [np.ones((1, 1), np.complex128)], [0.0]
        e, acc = envs[0], 0.0
        for k in range(self.n):
            a = self.sites[k]
            e = np.einsum("xsc,xsd->cd", a.conj(), np.einsum("xy,ysd->xsd", e, a))
            tr = float(np.real(np.trace(e)))
            if tr > 0:
                e = e / tr
                acc += math.log(tr)
            envs.append(e)
            logs.append(acc)
        return envs, logs

    def _transfer_right(self):
        envs, logs = [None] * (self.n + 1), [0.0] * (self.n + 1)
        envs[self.n] = np.ones((1, 1), np.complex128)
        e, acc = envs[self.n], 0.0
        for k in range(self.n - 1, -1, -1):
            a = self.sites[k]
            e = np.einsum("csx,dsx->cd", a.conj(), np.einsum("dsy,xy->dsx", a, e))
            tr = float(np.real(np.trace(e)))
            if tr > 0:
                e = e / tr
                acc += math.log(tr)
            envs[k] = e
            logs[k] = acc
        return envs, logs

    def norm_sq(self) -> float:
        """<psi|psi> including exp(2*norm_log)."""
        L, lg = self._transfer_left()
        return float(np.real(L[self.n][0, 0])) * math.exp(lg[self.n] + 2.0 * self.norm_log)

    def expect_local(self, ops: Dict[int, np.ndarray], envs=None) -> float:
        """Normalised <psi| prod_k O_k |psi> / <psi|psi> for operators on a contiguous site range."""
        sites = sorted(ops)
        lo, hi = sites[0], sites[-1]
        L, R = envs if envs is not None else (self._transfer_left()[0], self._transfer_right()[0])
        num, den = L[lo], L[lo]
        for k in range(lo, hi + 1):
            a = self.sites[k]
            op = ops.get(k, np.eye(2, dtype=np.complex128))
            num = np.einsum("xsc,xsd->cd", a.conj(), np.einsum("st,xy,ytd->xsd", op, num, a, optimize=True))
            den = np.einsum("xsc,xsd->cd", a.conj(), np.einsum("xy,ysd->xsd", den, a))
        val = np.einsum("cd,cd->", num, R[hi + 1])
        nrm = np.einsum("cd,cd->", den, R[hi + 1])
        return float(np.real(val / nrm))

    def environments(self):
        """(left, right) trace-normalised environments, reusable across expect_local calls."""
        return self._transfer_left()[0], self._transfer_right()[0]

    def expect_z_all(self) -> np.ndarray:
        z = np.diag([1.0, -1.0]).astype(np.complex128)
        envs = self.environments()
        return np.array([self.expect_local({k: z}, envs) for k in range(self.n)])

    # -- sampling (mps_core.py:354-429) -------------------------------------
    def right_environments(self) -> List[np.ndarray]:
        out: List[Optional[np.ndarray]] = [None] * (self.n + 1)
        out[self.n] = np.ones((1, 1), np.complex128)
        for k in range(self.n - 1, -1, -1):
            a = self.sites[k]
            # R_new[i, j] = sum_{s,b,c} A[i,s,b] R[b,c] conj(A[j,s,c])  (mps_core.py:364)
            e = np.einsum("isc,jsc->ij", np.einsum("isb,bc->isc", a, out[k + 1]), a.conj())
            tr = float(np.real(np.trace(e)))
            if tr > 1e-300:
                e = e / tr
            out[k] = e
        return out

    def sample(self, num_shots: int = 1, measured_qubits: Optional[Sequence[int]] = None,
               rng: Optional[np.random.Generator] = None) -> List[str]:
        """Sequential conditional sampling, mps_core.py:371-419 (one rng.choice per site and shot).

        A second positional argument that is a Generator is taken as ``rng``
        (the reference's signature is (num_shots, measured_qubits, rng)).  For a
        qubit subset the bitstring is built as bits[n-1-q] over the qubits in
        decreasing order, exactly as mps_core.py:414-416 does.
        """
        if isinstance(measured_qubits, np.random.Generator):
            measured_qubits, rng = None, measured_qubits
        if rng is None:
            rng = np.random.default_rng()
        envs = self.right_environments()
        shots = []
        for _ in range(num_shots):
            v = np.ones((1,), np.complex128)
            bits = []
            for k in range(self.n):
                a, e = self.sites[k], envs[k + 1]
                pr = np.zeros(2)
                for s in range(2):
                    w = v @ a[:, s, :]
                    pr[s] = float(np.real(w @ e @ w.conj()))
                pr = np.maximum(pr, 0.0)
                tot = pr.sum()
                pr = np.array([0.5, 0.5]) if tot < 1e-15 else pr / tot
                o = int(rng.choice(2, p=pr))
                bits.append(o)
                v = v @ a[:, o, :]
                nv = float(np.linalg.norm(v))
                if nv > 1e-15:
                    v = v / nv
            bs = "".join(str(b) for b in reversed(bits))
            if measured_qubits is not None and set(measured_qubits) != set(range(self.n)):
                ms = sorted(measured_qubits, reverse=True)
                bs = "".join(str(bits[self.n - 1 - q]) for q in ms)
            shots.append(bs)
        return shots


def mps_overlap(sites_a, sites_b, log_a: float = 0.0, log_b: float = 0.0):
    """<a|b> of two MPS given as lists of (chi_l, 2, chi_r) tensors, as
    (mantissa, log_scale) with <a|b> = mantissa * exp(log_scale); the norm_log
    factors of both states are included."""
    e = np.ones((1, 1), np.complex128)
    acc = 0.0
    for a, b in zip(sites_a, sites_b):
        e = np.einsum("xsc,xsd->cd", a.conj(), np.einsum("xy,ysd->xsd", e, b))
        s = float(np.max(np.abs(e)))
        if s > 0:
            e = e / s
            acc += math.log(s)
    return complex(e[0, 0]), acc + log_a + log_b


def infidelity(sites_a, sites_b) -> float:
    """1 - |<a|b>|^2 / (<a|a><b|b>) of two MPS (norm_log factors cancel)."""
    ab, lab = mps_overlap(sites_a, sites_b)
    aa, laa = mps_overlap(sites_a, sites_a)
    bb, lbb = mps_overlap(sites_b, sites_b)
    f = abs(ab) ** 2 / (aa.real * bb.real) * math.exp(2 * lab - laa - lbb)
    return float(1.0 - f)


# -- dense statevector helpers (exact references) ------------------------------
def dense_zero_state(n: int) -> np.ndarray:
    """|0...0> as an (2,)*n tensor with axis k = qubit k."""
    psi = np.zeros((2,) * n, dtype=np.complex128)
    psi[(0,) * n] = 1.0
    return psi


def dense_apply_1q(psi: np.ndarray, q: int, gate: np.ndarray) -> np.ndarray:
    return np.moveaxis(np.tensordot(gate, psi, axes=([1], [q])), 0, q)


def dense_apply_2q(psi: np.ndarray, qa: int, qb: int, gate: np.ndarray) -> np.ndarray:
    """Apply a 4x4 gate whose high index bit is qubit qa and low bit is qubit qb."""
    g = np.asarray(gate, np.complex128).reshape(2, 2, 2, 2)
    out = np.tensordot(g, psi, axes=([2, 3], [qa, qb]))
    return np.moveaxis(out, [0, 1], [qa, qb])


def dense_to_qiskit(psi: np.ndarray) -> np.ndarray:
    """Flatten with qubit 0 as the least significant bit."""
    n = psi.ndim
    return psi.transpose(list(range(n - 1, -1, -1))).reshape(-1)


def dense_expect_pauli(psi: np.ndarray, ops: Dict[int, np.ndarray]) -> float:
    phi = psi
    for q, op in ops.items():
        phi = dense_apply_1q(phi, q, op)
    return float(np.real(np.vdot(psi, phi) / np.vdot(psi, psi)))


def fidelity(a: np.ndarray, b: np.ndarray) -> float:
    """|<a|b>|^2 / (<a|a><b|b>)."""
    return float(abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real))


def haar_4x4_oracle(rng: np.random.Generator) -> np.ndarray:
    """Independent restatement of the Haar U(4) draw used by the workloads."""
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    ph = np.diagonal(r) / np.abs(np.diagonal(r))
    return q @ np.diag(ph)
