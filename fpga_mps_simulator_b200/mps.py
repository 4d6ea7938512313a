"""Device-resident MPS chains driven through libmpsb200 (no CPU fallback).

``MPSState`` mirrors the public surface of the reference class
``MPSState`` (mps_core.py:172-494): same constructor arguments, ``sites``,
``norm_log``, ``apply_1q``, ``apply_2q``, ``_apply_adjacent_2q``,
``get_statevector``, ``chi_l``/``chi_r``/``max_bond``/``bond_dims``,
``copy``.  It adds what the reference lacks for long chains --
``expectation``, ``amplitude`` and batched ``apply_layer`` -- with semantics
fixed by the reference's statevector convention (amplitudes carry
exp(norm_log); expectation values are normalised by <psi|psi>).

``MPSBatch`` holds many independent chains of uneven length and bond cap in
one allocation and advances them together, one launch per layer.

Storage (HBM): every site owns a slot of 2*chi_cap^2 complex128; site k is
kept C-order as (bonds[k], 2, bonds[k+1]) at the slot start.  Bond dimensions
live on the device and are written by the update kernel, so a sequence of
updates needs no host synchronisation.  Numerical faults (Jacobi not
converged, non-finite theta) are OR-ed into a per-chain device word that the
host checks whenever it reads results back (``check_status``).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, Iterable, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from .gates import GATE_MATRICES, permute_2q

__all__ = ["MPSState", "MPSBatch", "PairBatch", "FlowBatch", "PRECISIONS", "validate_pairs", "flow_items", "overlap",
           "infidelity"]

# "mixed": 3xTF32 tensor-core theta where it fills a 128-row tile (chi_cap > 32),
# the exact FP64 contraction below; "mixed_all": the tensor cores at every cap
# (64-row tiles at chi_cap <= 32).  Both: FP64 Jacobi SVD, 1e-6 S[0] floor.
PRECISIONS = {"fp64": _lib.FP64, "complex128": _lib.FP64, "mixed": _lib.MIXED_TF32X3,
              "tf32x3": _lib.MIXED_TF32X3, "mixed_all": _lib.TF32X3_ALL}
_SWAP = GATE_MATRICES["swap"]


def _stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def validate_pairs(ns: Sequence[int], chain_idx: np.ndarray, sites: np.ndarray) -> None:
    """Host check of one launch's pair table (the kernels trust it).

    Every pair (i, i+1) must lie inside its chain, the pairs of a chain must
    be disjoint, and all pairs of a chain must be contiguous in the table
    (the per-chain norm_log fold walks one contiguous run).
    """
    chain_idx = np.asarray(chain_idx, np.int64)
    sites = np.asarray(sites, np.int64)
    if len(chain_idx) != len(sites):
        raise ValueError("chain_idx and sites differ in length")
    if len(chain_idx) == 0:
        return
    if np.any(chain_idx < 0) or np.any(chain_idx >= len(ns)):
        raise ValueError("pair chain index out of range")
    nn = np.asarray(ns, np.int64)[chain_idx]
    if np.any(sites < 0) or np.any(sites + 1 >= nn):
        raise ValueError("pair site out of range: need 0 <= i and i + 1 < n")
    change = np.flatnonzero(np.diff(chain_idx) != 0)
    heads = chain_idx[np.concatenate([[0], change + 1])]
    if len(np.unique(heads)) != len(heads):
        raise ValueError("all pairs of one chain must be contiguous in the batch")
    order = np.lexsort((sites, chain_idx))
    cs, ss = chain_idx[order], sites[order]
    same = cs[1:] == cs[:-1]
    if np.any(same & (ss[1:] - ss[:-1] < 2)):
        raise ValueError("pairs of one launch must be disjoint")


def flow_items(ns: Sequence[int], chain_idx, sites) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Work list of the dataflow update launch from updates listed in application order.

    Item k is the update (chain_idx[k], sites[k]); a chain's updates apply in
    the order they appear.  Returns (items, order, offsets): items (K, 6) int32
    rows (chain, site, gate = k, out = k, dep0, dep1) where dep0 / dep1 are
    the last earlier items touching site i / site i+1 of the same chain (-1:
    none), so every dependency precedes its item (the topological order the
    kernel's forward progress rests on); order / offsets list each chain's
    items (CSR, chain c at order[offsets[c]:offsets[c+1]]) for the per-chain
    norm_log fold.
    """
    chain_idx = np.asarray(chain_idx, np.int64).reshape(-1)
    sites = np.asarray(sites, np.int64).reshape(-1)
    if len(chain_idx) != len(sites):
        raise ValueError("chain_idx and sites differ in length")
    K = len(sites)
    if K and (np.any(chain_idx < 0) or np.any(chain_idx >= len(ns))):
        raise ValueError("item chain index out of range")
    if K and (np.any(sites < 0) or np.any(sites + 1 >= np.asarray(ns, np.int64)[chain_idx])):
        raise ValueError("item site out of range: need 0 <= i and i + 1 < n")
    items = np.empty((K, 6), np.int32)
    last: Dict[Tuple[int, int], int] = {}
    for k in range(K):
        c, i = int(chain_idx[k]), int(sites[k])
        items[k] = (c, i, k, k, last.get((c, i), -1), last.get((c, i + 1), -1))
        last[(c, i)] = k
        last[(c, i + 1)] = k
    order = np.argsort(chain_idx, kind="stable").astype(np.int32)
    offsets = np.zeros(len(ns) + 1, np.int32)
    np.cumsum(np.bincount(chain_idx, minlength=len(ns)), out=offsets[1:])
    return items, order, offsets


class _Workspace:
    """Grow-only device scratch shared by the calls of one owner."""

    def __init__(self, device):
        self.device = device
        self.buf: Optional[torch.Tensor] = None

    def get(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self.buf


class PairBatch:
    """Device descriptor table for one launch of disjoint two-site updates.

    Built once on the host (validated: pairs in range, disjoint per chain,
    chains contiguous) and reusable across launches and CUDA-graph replays.
    """

    def __init__(self, owner: "MPSBatch", chain_idx: Sequence[int], sites: Sequence[int],
                 gates: np.ndarray, record_spectra: bool = False):
        chain_idx = np.asarray(chain_idx, dtype=np.int32)
        sites = np.asarray(sites, dtype=np.int32)
        if isinstance(gates, torch.Tensor):
            if gates.dtype != torch.complex128:
                raise ValueError("gates must be complex128")
            gates = gates.reshape(-1, 4, 4)
        else:
            gates = np.asarray(gates, dtype=np.complex128).reshape(-1, 4, 4)
        if not (len(chain_idx) == len(sites) == len(gates)):
            raise ValueError("chain_idx, sites and gates must have one entry per pair")
        owner._validate_pairs(chain_idx, sites)
        P = len(sites)
        self.npairs = P
        self.owner = owner
        dev = owner.device
        table = np.stack([chain_idx, sites, np.arange(P, dtype=np.int32), np.arange(P, dtype=np.int32)], 1)
        self.pairs = torch.from_numpy(np.ascontiguousarray(table)).to(dev)
        if isinstance(gates, torch.Tensor):  # e.g. pinned host memory: asynchronous copy
            self.gates = gates.reshape(P, 16).to(dev, non_blocking=True)
        else:
            self.gates = torch.from_numpy(np.ascontiguousarray(gates.reshape(P, 16))).to(dev)
        self.status = torch.zeros(P, dtype=torch.int32, device=dev)
        self.kept = torch.zeros(P, dtype=torch.int32, device=dev)
        self.trunc = torch.zeros(P, dtype=torch.float64, device=dev)
        self.spectra = torch.zeros(P, 128, dtype=torch.float64, device=dev) if record_spectra else None

    def set_gates(self, gates: np.ndarray) -> None:
        g = torch.from_numpy(np.ascontiguousarray(np.asarray(gates, np.complex128).reshape(self.npairs, 16)))
        self.gates.copy_(g, non_blocking=False)


class FlowBatch:
    """Device work list for one dataflow launch: many layers of many chains.

    ``chain_idx``, ``sites``, ``gates`` list updates in application order
    (e.g. layer by layer); outputs (status, kept, trunc, spectra) have one row
    per item.  Reusable across launches and CUDA-graph replays.
    """

    def __init__(self, owner: "MPSBatch", chain_idx, sites, gates, record_spectra: bool = False):
        items, order, offsets = flow_items(owner.ns, chain_idx, sites)
        dev = owner.device
        self.owner = owner
        self.nitems = len(items)
        self.items = torch.from_numpy(np.ascontiguousarray(items)).to(dev)
        self.order = torch.from_numpy(order).to(dev)
        self.offsets = torch.from_numpy(offsets).to(dev)
        self.gates = torch.empty(self.nitems, 16, dtype=torch.complex128, device=dev)
        self.set_gates(gates)
        self.status = torch.zeros(self.nitems, dtype=torch.int32, device=dev)
        self.kept = torch.zeros(self.nitems, dtype=torch.int32, device=dev)
        self.trunc = torch.zeros(self.nitems, dtype=torch.float64, device=dev)
        self.spectra = torch.zeros(self.nitems, 128, dtype=torch.float64, device=dev) if record_spectra else None
        self.host_items = items

    def set_gates(self, gates) -> None:
        """Replace the gates (one 4x4 per item, list order): a numpy array, or a
        torch tensor -- from pinned host memory the copy is asynchronous."""
        if isinstance(gates, torch.Tensor):
            if gates.dtype != torch.complex128 or gates.numel() != 16 * self.nitems:
                raise ValueError("gates must be complex128 with one 4x4 per item")
            self.gates.copy_(gates.reshape(self.nitems, 16), non_blocking=True)
            return
        g = np.asarray(gates, dtype=np.complex128)
        if g.size != 16 * self.nitems:
            raise ValueError("need one gate per item")
        self.gates.copy_(torch.from_numpy(np.ascontiguousarray(g.reshape(self.nitems, 16))))


class ThetaBatch:
    """Device tables for one contraction-only launch (``MPSBatch.run_thetas``).

    Pair k is (chain_idx[k], sites[k]) with gate k; pairs only read the sites,
    so they may overlap.  ``theta`` holds one (2 chi_cap)^2 row per pair: the
    (2 chi_l) x (2 chi_r) matrix, row-major, at its start.  Reusable across
    launches and CUDA-graph replays.
    """

    def __init__(self, owner: "MPSBatch", chain_idx, sites, gates):
        chain_idx = np.asarray(chain_idx, np.int64).reshape(-1)
        sites = np.asarray(sites, np.int64).reshape(-1)
        g = np.asarray(gates, dtype=np.complex128).reshape(-1, 16)
        if not (len(chain_idx) == len(sites) == len(g)):
            raise ValueError("chain_idx, sites and gates must have one entry per pair")
        P = len(sites)
        if P and (np.any(chain_idx < 0) or np.any(chain_idx >= owner.nchains)):
            raise ValueError("pair chain index out of range")
        if P and (np.any(sites < 0) or np.any(sites + 1 >= np.asarray(owner.ns, np.int64)[chain_idx])):
            raise ValueError("pair site out of range: need 0 <= i and i + 1 < n")
        dev = owner.device
        self.owner = owner
        self.npairs = P
        self.chain_idx = chain_idx
        self.sites = sites
        table = np.stack([chain_idx, sites, np.arange(P), np.arange(P)], 1).astype(np.int32)
        self.pairs = torch.from_numpy(np.ascontiguousarray(table)).to(dev)
        self.gates = torch.from_numpy(np.ascontiguousarray(g)).to(dev)
        self.status = torch.zeros(P, dtype=torch.int32, device=dev)
        self.theta = torch.zeros(P, (2 * owner.chi_cap) ** 2, dtype=torch.complex128, device=dev)

    def matrices(self) -> List[np.ndarray]:
        """Host copies of the thetas, each (2 chi_l, 2 chi_r), from the current bonds."""
        th = self.theta.cpu().numpy()
        bonds = self.owner.bonds.cpu().numpy()
        out = []
        for k in range(self.npairs):
            c, i = int(self.chain_idx[k]), int(self.sites[k])
            b0 = int(self.owner.bond_off[c])
            cl, cr = int(bonds[b0 + i]), int(bonds[b0 + i + 2])
            out.append(th[k, : 4 * cl * cr].reshape(2 * cl, 2 * cr).copy())
        return out


class MPSBatch:
    """Independent chains in one device allocation.

    ``ns[c]``, ``chi_maxs[c]``, ``cutoffs[c]`` give chain c's length, bond
    cap and relative SVD cutoff.  All chains start in |0...0>.
    """

    def __init__(self, ns: Sequence[int], chi_maxs: Union[int, Sequence[int]] = 64,
                 cutoffs: Union[float, Sequence[float]] = 1e-12, precision: str = "fp64",
                 device: Union[str, torch.device] = "cuda", tol: float = 0.0, max_sweeps: int = 0):
        ns = [int(v) for v in ns]
        nch = len(ns)
        chi_maxs = [int(chi_maxs)] * nch if np.isscalar(chi_maxs) else [int(v) for v in chi_maxs]
        cutoffs = [float(cutoffs)] * nch if np.isscalar(cutoffs) else [float(v) for v in cutoffs]
        if nch == 0 or len(chi_maxs) != nch or len(cutoffs) != nch:
            raise ValueError("need one n, chi_max and cutoff per chain")
        for n, chi in zip(ns, chi_maxs):
            if n < 1:
                raise ValueError(f"chain length must be >= 1, got {n}")
            if chi < 1:
                raise ValueError(f"chi_max must be >= 1, got {chi}")
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("MPSBatch lives on a CUDA device; there is no CPU engine")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _lib.OnDevice(_lib.load(), self.device)
        self.precision = precision
        self.tol = float(tol)
        self.max_sweeps = int(max_sweeps)
        self.ns = ns
        self.chi_maxs = chi_maxs
        self.cutoffs = cutoffs
        # device bond cap per chain: min(chi_max, MPSB_CHI_LIMIT, 2^(n//2)); a chain
        # whose chi_max exceeds the limit reports MPSB_ST_CHI_LIMIT from the first
        # update that would keep more than the limit
        self.caps = [_lib.keep_limit(n, chi) for n, chi in zip(ns, chi_maxs)]
        self.chi_cap = max(self.caps)
        self.slot = 2 * self.chi_cap * self.chi_cap
        self.site_off = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
        self.bond_off = self.site_off + np.arange(nch + 1)
        dev = self.device
        total = int(self.site_off[-1])
        self.sites = torch.zeros(total, self.slot, dtype=torch.complex128, device=dev)
        self.sites[:, 0] = 1.0
        self.bonds = torch.ones(total + nch, dtype=torch.int32, device=dev)
        self.norm_logs = torch.zeros(nch, dtype=torch.float64, device=dev)
        self.status_acc = torch.zeros(nch, dtype=torch.int32, device=dev)
        self._ws = _Workspace(dev)
        self._ews = _Workspace(dev)
        self._build_table()

    # -- chain table ----------------------------------------------------------
    def _build_table(self) -> None:
        self.table = self.make_table(self.sites, self.bonds)

    def make_table(self, sites: torch.Tensor, bonds: torch.Tensor) -> torch.Tensor:
        """Device chain table over ``sites`` / ``bonds`` laid out like this batch's own
        (used for saved copies of the state and for cotangent arrays)."""
        if sites.shape != self.sites.shape or bonds.shape != self.bonds.shape:
            raise ValueError("a chain table needs sites and bonds shaped like the batch's")
        nch = len(self.ns)
        arr = (_lib.Chain * nch)()
        sb = sites.element_size() * self.slot
        for c in range(nch):
            arr[c].sites = sites.data_ptr() + int(self.site_off[c]) * sb
            arr[c].bonds = bonds.data_ptr() + int(self.bond_off[c]) * 4
            arr[c].norm_log = self.norm_logs.data_ptr() + c * 8
            arr[c].status_acc = self.status_acc.data_ptr() + c * 4
            arr[c].slot_elems = self.slot
            arr[c].n = self.ns[c]
            arr[c].chi_max = self.chi_maxs[c]
            arr[c].cutoff = self.cutoffs[c]
        raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
        return torch.from_numpy(raw).to(self.device)

    def chain_ptr(self, c: int) -> int:
        return self.table.data_ptr() + c * C.sizeof(_lib.Chain)

    @property
    def nchains(self) -> int:
        return len(self.ns)

    def _stream(self) -> int:
        return _stream_handle(self.device)

    def _validate_pairs(self, chain_idx: np.ndarray, sites: np.ndarray) -> None:
        validate_pairs(self.ns, chain_idx, sites)

    # -- updates --------------------------------------------------------------
    def make_pairs(self, chain_idx, sites, gates, record_spectra: bool = False) -> PairBatch:
        return PairBatch(self, chain_idx, sites, gates, record_spectra)

    def run_pairs(self, pb: PairBatch, precision: Optional[str] = None, chi_cap: Optional[int] = None,
                  workspace: Optional[_Workspace] = None, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Launch one batched update (asynchronous, stream-ordered, graph-capturable).

        ``chi_cap`` may be lowered to the largest chi_max of the chains this
        launch touches (smaller shared memory per CTA); launches running
        concurrently on different ``stream``s need their own ``workspace``.
        """
        if pb.npairs == 0:
            return
        prec = PRECISIONS[precision or self.precision]
        cap = self.chi_cap if chi_cap is None else int(chi_cap)
        need = self._lib.mpsb_update2q_workspace_bytes(pb.npairs, cap)
        ws = (workspace or self._ws).get(need)
        handle = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        rc = self._lib.mpsb_update2q_batch(
            self.table.data_ptr(), pb.pairs.data_ptr(), pb.npairs, pb.gates.data_ptr(), prec,
            cap, self.tol, self.max_sweeps, ws.data_ptr(), ws.numel(),
            _ptr(pb.spectra), pb.kept.data_ptr(), pb.trunc.data_ptr(), pb.status.data_ptr(), handle)
        _lib.check(rc, "mpsb_update2q_batch")

    def make_thetas(self, chain_idx, sites, gates) -> ThetaBatch:
        return ThetaBatch(self, chain_idx, sites, gates)

    def run_thetas(self, tb: ThetaBatch, precision: Optional[str] = None,
                   stream: Optional[torch.cuda.Stream] = None) -> None:
        """theta = G (A B) of every pair of ``tb``, no SVD (asynchronous, stream-ordered).

        The contraction the update of ``precision`` runs at this batch's bond
        cap (``mpsb_contract2q_batch``): the device half of the reference's
        FPGA offload, fpga_mps_simulator.cpp:287-371.  Status bits per pair
        land in ``tb.status``.
        """
        if tb.npairs == 0:
            return
        prec = PRECISIONS[precision or self.precision]
        handle = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        rc = self._lib.mpsb_contract2q_batch(
            self.table.data_ptr(), tb.pairs.data_ptr(), tb.npairs, tb.gates.data_ptr(), prec, self.chi_cap,
            tb.theta.data_ptr(), tb.status.data_ptr(), handle)
        _lib.check(rc, "mpsb_contract2q_batch")

    def thetas(self, chain_idx, sites, gates, precision: Optional[str] = None) -> List[np.ndarray]:
        """Host thetas, (2 chi_l, 2 chi_r) each, of the given pairs (synchronous)."""
        tb = self.make_thetas(chain_idx, sites, gates)
        self.run_thetas(tb, precision)
        st = tb.status.cpu().numpy()
        if np.any(st):
            raise RuntimeError("contraction failed: " + "; ".join(
                f"pair {k}: {_lib.status_text(int(v))}" for k, v in enumerate(st) if v))
        return tb.matrices()

    def make_flow(self, chain_idx, sites, gates, record_spectra: bool = False) -> FlowBatch:
        return FlowBatch(self, chain_idx, sites, gates, record_spectra)

    def run_flow(self, fb: FlowBatch, precision: Optional[str] = None, chi_cap: Optional[int] = None,
                 threads: int = 0, nclusters: int = 0, poll_limit: int = -1,
                 workspace: Optional[_Workspace] = None, stream: Optional[torch.cuda.Stream] = None) -> None:
        """One dataflow launch over the whole work list (asynchronous, graph-capturable).

        ``threads`` picks the CTA shape (0 = default for the cap), ``nclusters``
        the number of workspace slots, i.e. concurrently working clusters
        (0 = all that fit), ``poll_limit`` the polls per dependency wait
        (-1 = the library default).
        """
        if fb.nitems == 0:
            return
        prec = PRECISIONS[precision or self.precision]
        cap = self.chi_cap if chi_cap is None else int(chi_cap)
        need = self._lib.mpsb_update2q_flow_workspace_bytes(fb.nitems, cap, prec, int(threads), int(nclusters))
        if need == 0:
            _lib.check(-1, "mpsb_update2q_flow_workspace_bytes")
        ws = (workspace or self._ws).get(need)
        handle = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        rc = self._lib.mpsb_update2q_flow(
            self.table.data_ptr(), self.nchains, fb.items.data_ptr(), fb.nitems, fb.order.data_ptr(),
            fb.offsets.data_ptr(), fb.gates.data_ptr(), prec, cap, self.tol, self.max_sweeps, int(threads),
            int(nclusters), int(poll_limit), ws.data_ptr(), ws.numel(), _ptr(fb.spectra), fb.kept.data_ptr(),
            fb.trunc.data_ptr(), fb.status.data_ptr(), handle)
        _lib.check(rc, "mpsb_update2q_flow")

    def snapshot(self):
        """Device copies of the mutable state (sites, bonds, norm_log, status)."""
        return (self.sites.clone(), self.bonds.clone(), self.norm_logs.clone(), self.status_acc.clone())

    def restore(self, snap) -> None:
        self.sites.copy_(snap[0])
        self.bonds.copy_(snap[1])
        self.norm_logs.copy_(snap[2])
        self.status_acc.copy_(snap[3])

    def apply_layer(self, chain_idx, sites, gates, precision: Optional[str] = None,
                    record_spectra: bool = False) -> PairBatch:
        pb = self.make_pairs(chain_idx, sites, gates, record_spectra)
        self.run_pairs(pb, precision)
        return pb

    def apply_1q_many(self, chain_idx, sites, gates) -> None:
        chain_idx = np.asarray(chain_idx, np.int32)
        sites = np.asarray(sites, np.int32)
        g = np.asarray(gates, np.complex128).reshape(-1, 4)
        if len(sites) == 0:
            return
        key = chain_idx.astype(np.int64) * (1 << 32) + sites
        if len(np.unique(key)) != len(key):
            raise ValueError("single-site ops of one launch must touch distinct sites")
        if np.any(sites < 0) or np.any(sites >= np.asarray(self.ns)[chain_idx]):
            raise ValueError("site out of range")
        ops = np.stack([chain_idx, sites, np.arange(len(sites), dtype=np.int32),
                        np.zeros(len(sites), np.int32)], 1)
        ops_t = torch.from_numpy(np.ascontiguousarray(ops)).to(self.device)
        g_t = torch.from_numpy(np.ascontiguousarray(g)).to(self.device)
        rc = self._lib.mpsb_apply1q_batch(self.table.data_ptr(), ops_t.data_ptr(), len(sites),
                                          g_t.data_ptr(), self.chi_cap, self._stream())
        _lib.check(rc, "mpsb_apply1q_batch")

    # -- read-out -------------------------------------------------------------
    def check_status(self, raise_on_error: bool = True) -> np.ndarray:
        st = self.status_acc.cpu().numpy()
        if raise_on_error and np.any(st):
            bad = {int(c): f"{int(v)} ({_lib.status_text(int(v))})" for c, v in enumerate(st) if v}
            hint = ""
            if any(int(v) & _lib.ST_CHI_LIMIT for v in st):
                hint = (f"; this device path forms bonds of at most {_lib.MPSB_CHI_LIMIT}, so an update whose "
                        f"chi_max allows more cannot follow mps_core: pass chi_max <= {_lib.MPSB_CHI_LIMIT} to "
                        "truncate there")
            raise RuntimeError(f"two-site update reported faults per chain {bad}{hint}")
        return st

    def bond_dims(self, c: int = 0) -> List[int]:
        b = self.bonds[int(self.bond_off[c]): int(self.bond_off[c]) + self.ns[c] + 1].cpu().numpy()
        return [int(v) for v in b[1:-1]]

    def norm_log(self, c: int = 0) -> float:
        return float(self.norm_logs[c].item())

    def site(self, c: int, k: int) -> np.ndarray:
        b = self.bonds[int(self.bond_off[c]) + k: int(self.bond_off[c]) + k + 2].cpu().numpy()
        flat = self.sites[int(self.site_off[c]) + k, : b[0] * 2 * b[1]].cpu().numpy()
        return flat.reshape(int(b[0]), 2, int(b[1])).copy()

    def set_site(self, c: int, k: int, tensor) -> None:
        t = np.asarray(tensor, dtype=np.complex128)
        if t.ndim != 3 or t.shape[1] != 2:
            raise ValueError("site tensor must have shape (chi_l, 2, chi_r)")
        n = self.ns[c]
        bl, br = self.bonds[int(self.bond_off[c]) + k: int(self.bond_off[c]) + k + 2].cpu().numpy()
        if (k == 0 and t.shape[0] != 1) or (k == n - 1 and t.shape[2] != 1):
            raise ValueError("boundary bonds must be 1")
        if max(t.shape[0], t.shape[2]) > self.chi_maxs[c]:
            raise ValueError("bond dimension above chi_max")
        if max(t.shape[0], t.shape[2]) > self.caps[c]:
            raise ValueError(f"bond dimension above the device limit {self.caps[c]}")
        # a bond can never exceed the Schmidt rank bound 2^min(left sites, right sites)
        if t.shape[0] > 2 ** min(k, n - k) or t.shape[2] > 2 ** min(k + 1, n - k - 1):
            raise ValueError("bond dimension above the Schmidt-rank bound of its cut")
        row = torch.zeros(self.slot, dtype=torch.complex128)
        row[: t.size] = torch.from_numpy(t.reshape(-1))
        self.sites[int(self.site_off[c]) + k].copy_(row.to(self.device))
        self.bonds[int(self.bond_off[c]) + k] = int(t.shape[0])
        self.bonds[int(self.bond_off[c]) + k + 1] = int(t.shape[2])

    def statevector(self, c: int = 0) -> np.ndarray:
        n = self.ns[c]
        if n > 24:
            raise ValueError(f"Statevector reconstruction for n={n} > 24 not supported.")
        out = torch.empty(1 << n, dtype=torch.complex128, device=self.device)
        scratch = torch.empty(2 << n, dtype=torch.complex128, device=self.device)
        rc = self._lib.mpsb_statevector(self.chain_ptr(c), n, self.chi_cap, out.data_ptr(), scratch.data_ptr(),
                                        scratch.numel() * 16, self._stream())
        _lib.check(rc, "mpsb_statevector")
        return out.cpu().numpy()

    def amplitudes(self, c: int, bits: np.ndarray, with_log: bool = False):
        bits = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8).reshape(-1, self.ns[c]))
        nb = bits.shape[0]
        bt = torch.from_numpy(bits).to(self.device)
        out = torch.empty(nb, dtype=torch.complex128, device=self.device)
        la = torch.empty(nb, dtype=torch.float64, device=self.device)
        rc = self._lib.mpsb_amplitude(self.table.data_ptr(), c, self.ns[c], bt.data_ptr(), nb, self.chi_cap,
                                      out.data_ptr(), la.data_ptr(), self._stream())
        _lib.check(rc, "mpsb_amplitude")
        return (out.cpu().numpy(), la.cpu().numpy()) if with_log else out.cpu().numpy()

    def sample_bits(self, c: int, uniforms: np.ndarray) -> np.ndarray:
        """Shots of chain c as a (shots, n) uint8 array (column i = qubit i).

        ``uniforms`` (shots, n) in [0, 1) drive the draws in (shot, site)
        order, one per draw, as the reference's per-site rng.choice does.
        """
        n = self.ns[c]
        u = np.ascontiguousarray(np.asarray(uniforms, np.float64).reshape(-1, n))
        shots = u.shape[0]
        if shots == 0:
            return np.zeros((0, n), np.uint8)
        ut = torch.from_numpy(u).to(self.device)
        bits = torch.empty(shots, n, dtype=torch.uint8, device=self.device)
        need = self._lib.mpsb_sample_workspace_bytes(n, self.chi_cap)
        ws = self._ews.get(need)
        rc = self._lib.mpsb_sample(self.table.data_ptr(), c, n, self.chi_cap, ut.data_ptr(), shots, bits.data_ptr(),
                                   ws.data_ptr(), ws.numel(), self._stream())
        _lib.check(rc, "mpsb_sample")
        return bits.cpu().numpy()

    def reset_many(self, chain_idx, sites) -> None:
        """Reset of fpga_mps_simulator.py:530-552 on distinct (chain, site) pairs, one launch."""
        chain_idx = np.asarray(chain_idx, np.int32).reshape(-1)
        sites = np.asarray(sites, np.int32).reshape(-1)
        if len(sites) == 0:
            return
        if np.any(sites < 0) or np.any(sites >= np.asarray(self.ns)[chain_idx]):
            raise ValueError("site out of range")
        key = chain_idx.astype(np.int64) * (1 << 32) + sites
        if len(np.unique(key)) != len(key):
            raise ValueError("reset sites of one launch must be distinct")
        ops = np.stack([chain_idx, sites, np.zeros_like(sites), np.zeros_like(sites)], 1)
        ops_t = torch.from_numpy(np.ascontiguousarray(ops)).to(self.device)
        rc = self._lib.mpsb_reset_batch(self.table.data_ptr(), ops_t.data_ptr(), len(sites), self.chi_cap,
                                        self._stream())
        _lib.check(rc, "mpsb_reset_batch")

    def canonicalize(self, chains: Sequence[int], lo: int, hi: int, direction: str = "left") -> None:
        """QR sweeps on the listed chains: "left" = left_normalize_site(i) for
        i = lo..hi, "right" = right_normalize_site(i) for i = hi..lo
        (mps_core.py:221-252), one launch."""
        chains = [int(c) for c in chains]
        if not chains or hi < lo:
            return
        if lo < 0 or any(hi >= self.ns[c] for c in chains):
            raise ValueError("canonicalisation range outside a chain")
        if direction not in ("left", "right"):
            raise ValueError("direction must be 'left' or 'right'")
        ids = torch.tensor(chains, dtype=torch.int32, device=self.device)
        need = self._lib.mpsb_canonicalize_workspace_bytes(len(chains), self.chi_cap)
        ws = self._ews.get(need)
        rc = self._lib.mpsb_canonicalize(self.table.data_ptr(), ids.data_ptr(), len(chains), int(lo), int(hi),
                                         0 if direction == "left" else 1, self.chi_cap, ws.data_ptr(), ws.numel(),
                                         self._stream())
        _lib.check(rc, "mpsb_canonicalize")

    def expect_terms(self, terms: Sequence[Tuple[int, np.ndarray, Optional[np.ndarray]]],
                     chains: Optional[Sequence[int]] = None) -> np.ndarray:
        """Normalised <O> for terms (site, O_site, O_next or None) on chains 0..nchains-1.

        All chains evaluated together must have the same length; returns
        (nchains, nterms).
        """
        nch = self.nchains if chains is None else len(chains)
        if chains is not None and list(chains) != list(range(nch)):
            raise ValueError("expect_terms evaluates a leading range of chains")
        n = self.ns[0]
        if any(self.ns[c] != n for c in range(nch)):
            raise ValueError("chains evaluated together must have equal length")
        sites = np.array([t[0] for t in terms], np.int32)
        two = np.array([0 if t[2] is None else 1 for t in terms], np.int32)
        if np.any(sites < 0) or np.any(sites + two >= n):
            raise ValueError("term site out of range")
        ops = np.zeros((len(terms), 2, 4), np.complex128)
        for k, (_, o1, o2) in enumerate(terms):
            ops[k, 0] = np.asarray(o1, np.complex128).reshape(4)
            ops[k, 1] = np.eye(2).reshape(4) if o2 is None else np.asarray(o2, np.complex128).reshape(4)
        dev = self.device
        st, tt, ot = (torch.from_numpy(sites).to(dev), torch.from_numpy(two).to(dev),
                      torch.from_numpy(ops.reshape(-1)).to(dev))
        out = torch.empty(nch * len(terms), dtype=torch.float64, device=dev)
        need = self._lib.mpsb_expect_workspace_bytes(nch, n, self.chi_cap)
        ws = self._ews.get(need)
        rc = self._lib.mpsb_expect_local(self.table.data_ptr(), nch, n, self.chi_cap, st.data_ptr(),
                                         tt.data_ptr(), ot.data_ptr(), len(terms), out.data_ptr(),
                                         ws.data_ptr(), ws.numel(), self._stream())
        _lib.check(rc, "mpsb_expect_local")
        return out.cpu().numpy().reshape(nch, len(terms))


def overlap(a: "MPSBatch", ca: int, b: "MPSBatch", cb: int) -> Tuple[complex, float]:
    """<a_ca | b_cb> as (mantissa, log_scale), norm_log of both chains included."""
    if a.ns[ca] != b.ns[cb]:
        raise ValueError("overlap needs chains of equal length")
    cap = max(a.chi_cap, b.chi_cap)
    out = torch.empty(1, dtype=torch.complex128, device=a.device)
    lg = torch.empty(1, dtype=torch.float64, device=a.device)
    ws = torch.empty(2 * cap * cap * 16, dtype=torch.uint8, device=a.device)
    rc = a._lib.mpsb_overlap(a.chain_ptr(ca), b.chain_ptr(cb), a.ns[ca], cap, out.data_ptr(), lg.data_ptr(),
                             ws.data_ptr(), ws.numel(), _stream_handle(a.device))
    _lib.check(rc, "mpsb_overlap")
    return complex(out.item()), float(lg.item())


def infidelity(a: "MPSState", b: "MPSState") -> float:
    """1 - |<a|b>|^2 / (<a|a><b|b>) of two single-chain states, on the device."""
    ab, lab = overlap(a._b, 0, b._b, 0)
    aa, laa = overlap(a._b, 0, a._b, 0)
    bb, lbb = overlap(b._b, 0, b._b, 0)
    return 1.0 - abs(ab) ** 2 / (aa.real * bb.real) * math.exp(2 * lab - laa - lbb)


_PAULI = {"I": np.eye(2, dtype=np.complex128), "X": GATE_MATRICES["x"], "Y": GATE_MATRICES["y"],
          "Z": GATE_MATRICES["z"]}


class _SitesView:
    """List-like access to the device site tensors: host copies on read, uploads on write."""

    def __init__(self, st: "MPSState"):
        self._st = st

    def __len__(self):
        return self._st.n

    def __getitem__(self, k):
        if isinstance(k, slice):
            return [self[j] for j in range(*k.indices(len(self)))]
        if k < 0:
            k += len(self)
        if not 0 <= k < len(self):
            raise IndexError(k)
        return self._st._b.site(0, k)

    def __setitem__(self, k, value):
        self._st._b.set_site(0, k, value)

    def __iter__(self):
        return (self[k] for k in range(len(self)))


class MPSState:
    """One MPS chain on the GPU with the reference class's interface.

    Parameters follow mps_core.MPSState(n, chi_max=256, svd_cutoff=1e-12)
    (mps_core.py:185), defaults included.  The device forms bonds of at most
    64 (theta <= 128 x 128 on chip; the reference's FPGA build caps chi the
    same way, fpga_mps_simulator.py:80-85).  Any chi_max is accepted: while no
    update would keep more than 64 values -- always for n <= 12, where no
    bond can exceed 64 -- the state follows mps_core exactly; an update that
    would keep more marks the chain (status MPSB_ST_CHI_LIMIT) and every
    read-out then raises instead of returning a state that differs from the
    reference's.  ``precision`` selects the FP64 drop-in form or the mixed
    3xTF32 form.

    Gate-by-gate use, as mps_core callers write it: ``_apply_adjacent_2q`` /
    ``apply_2q`` calls are queued (``defer=True``, the default) and run as
    ONE dataflow launch when the state is next read or changed in another
    way, or when ``flush_at`` updates are waiting: each update starts as soon
    as the earlier updates on its two sites are done, so disjoint gates of a
    circuit run side by side instead of one 2-CTA cluster at a time.  The
    result is bit-identical to applying them one by one (``defer=False``).
    Argument errors still raise at the call.
    """

    def __init__(self, n: int, chi_max: int = 256, svd_cutoff: float = 1e-12, precision: str = "fp64",
                 device: Union[str, torch.device] = "cuda", tol: float = 0.0, max_sweeps: int = 0,
                 defer: bool = True, flush_at: int = 4096):
        self.n = int(n)
        self.chi_max = int(chi_max)
        self.svd_cutoff = float(svd_cutoff)
        self._batch = MPSBatch([self.n], [self.chi_max], [self.svd_cutoff], precision, device, tol, max_sweeps)
        self.precision = precision
        self.defer = bool(defer)
        self.flush_at = int(flush_at)
        self._pending: List[Tuple[int, np.ndarray]] = []
        self._last_pairs: Optional[PairBatch] = None
        self.last_flow: Optional[FlowBatch] = None

    @property
    def _b(self) -> MPSBatch:
        """The device batch, with every queued update applied first."""
        if self._pending:
            self.flush()
        return self._batch

    def flush(self) -> None:
        """Launch the queued two-site updates (one dataflow launch; asynchronous)."""
        if not self._pending:
            return
        sites = np.array([p[0] for p in self._pending], np.int32)
        gates = np.stack([p[1] for p in self._pending])
        self._pending = []
        self.last_flow = self._batch.make_flow(np.zeros(len(sites), np.int32), sites, gates)
        self._batch.run_flow(self.last_flow)

    @property
    def last_pairs(self) -> Optional[PairBatch]:
        """Per-update outputs of the last ``apply_layer`` (or undeferred update)."""
        self.flush()
        return self._last_pairs

    @last_pairs.setter
    def last_pairs(self, pb: Optional[PairBatch]) -> None:
        self._last_pairs = pb

    @property
    def device(self) -> torch.device:
        return self._batch.device

    # -- state -------------------------------------------------------------
    @property
    def sites(self) -> _SitesView:
        return _SitesView(self)

    @sites.setter
    def sites(self, tensors) -> None:
        tensors = list(tensors)
        if len(tensors) != self.n:
            raise ValueError("need one tensor per site")
        for k, t in enumerate(tensors):
            self._b.set_site(0, k, t)

    @property
    def norm_log(self) -> float:
        return self._b.norm_log(0)

    @norm_log.setter
    def norm_log(self, value: float) -> None:
        self._b.norm_logs[0] = float(value)

    def copy(self) -> "MPSState":
        out = MPSState(self.n, self.chi_max, self.svd_cutoff, self.precision, self.device,
                       self._b.tol, self._b.max_sweeps, self.defer, self.flush_at)
        out._b.sites.copy_(self._b.sites)
        out._b.bonds.copy_(self._b.bonds)
        out._b.norm_logs.copy_(self._b.norm_logs)
        out._b.status_acc.copy_(self._b.status_acc)
        return out

    def chi_l(self, i: int) -> int:
        return 1 if i == 0 else self.bond_dims()[i - 1]

    def chi_r(self, i: int) -> int:
        return 1 if i == self.n - 1 else self.bond_dims()[i]

    def bond_dims(self) -> List[int]:
        return self._b.bond_dims(0)

    def max_bond(self) -> int:
        return max(self.bond_dims()) if self.n > 1 else 1

    def check_status(self, raise_on_error: bool = True) -> int:
        return int(self._b.check_status(raise_on_error)[0])

    # -- gates -------------------------------------------------------------
    def apply_1q(self, site: int, gate: np.ndarray) -> None:
        """A'[l, s', r] = sum_s G[s', s] A[l, s, r] (mps_core.py:267-273)."""
        self._b.apply_1q_many([0], [int(site)], np.asarray(gate, np.complex128).reshape(1, 2, 2))

    def _apply_adjacent_2q(self, i: int, gate: np.ndarray) -> None:
        """contract -> gate -> truncated SVD -> sqrt(S) split on (i, i+1) (mps_core.py:326-350).

        Queued when ``defer`` is set (see the class notes); the gate is copied
        at the call."""
        i = int(i)
        if not 0 <= i < self.n - 1:
            raise ValueError(f"pair site out of range: need 0 <= i and i + 1 < n, got i={i}, n={self.n}")
        g = np.array(gate, dtype=np.complex128).reshape(4, 4)
        if not self.defer:
            self.last_pairs = self._b.apply_layer([0], [i], g[None])
            return
        self._pending.append((i, g))
        if len(self._pending) >= self.flush_at:
            self.flush()

    apply_adjacent_2q = _apply_adjacent_2q

    def theta(self, i: int, gate: np.ndarray) -> np.ndarray:
        """theta = G (A_i A_{i+1}) as the (2 chi_l, 2 chi_r) matrix the update would
        factorise, without applying it: what the reference's FPGA kernel returns
        for its host SVD (fpga_mps_simulator.py:584-600)."""
        i = int(i)
        if not 0 <= i < self.n - 1:
            raise ValueError(f"pair site out of range: need 0 <= i and i + 1 < n, got i={i}, n={self.n}")
        g = np.array(gate, dtype=np.complex128).reshape(1, 4, 4)
        return self._b.thetas([0], [i], g)[0]

    def apply_2q(self, i: int, j: int, gate: np.ndarray) -> None:
        """Dispatch of mps_core.py:304-324, including its SWAP routing.

        Non-adjacent (i, j) is routed with SWAPs and the gate applied on
        (lo, lo+1) as given (the reference does not re-index it); an adjacent
        pair given as (i+1, i) re-indexes the gate with [0, 2, 1, 3].
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
            g = permute_2q(g)
        self._apply_adjacent_2q(i, g)

    def apply_layer(self, sites: Sequence[int], gates: np.ndarray, record_spectra: bool = False) -> PairBatch:
        """All disjoint adjacent pairs (i, i+1), i in ``sites``, in one launch."""
        self.last_pairs = self._b.apply_layer(np.zeros(len(sites), np.int32), sites, gates,
                                              record_spectra=record_spectra)
        return self.last_pairs

    def apply_layers(self, layer_sites: Sequence[Sequence[int]], gates,
                     flow: Optional[FlowBatch] = None) -> FlowBatch:
        """Many layers of adjacent pairs in ONE dataflow launch.

        ``layer_sites[L]`` lists the left sites of layer L; ``gates`` holds one
        4x4 per pair in layer order (numpy, or a torch tensor, e.g. in pinned
        host memory).  Updates apply in that order -- the result is
        bit-identical to ``apply_layer`` for each layer in turn -- but each
        pair starts as soon as the two updates before it on its sites are
        done.  Passing the FlowBatch a previous call returned (same layers)
        reuses its device tables and only copies the new gates.
        """
        if flow is None:
            sites = np.concatenate([np.asarray(s, np.int32).reshape(-1) for s in layer_sites]) \
                if len(layer_sites) else np.zeros(0, np.int32)
            for s in layer_sites:  # each layer disjoint, as a layer of apply_layer must be
                validate_pairs([self.n], np.zeros(len(s), np.int64), np.asarray(s, np.int64))
            flow = self._b.make_flow(np.zeros(len(sites), np.int32), sites,
                                     np.zeros((len(sites), 4, 4), np.complex128))
        if flow.owner is not self._b:
            raise ValueError("the flow belongs to another state")
        flow.set_gates(gates)
        self._b.run_flow(flow)
        self.last_flow = flow
        return flow

    # -- read-out ------------------------------------------------------------
    def get_statevector(self) -> np.ndarray:
        """Dense amplitudes in Qiskit order including exp(norm_log) (mps_core.py:433-461)."""
        self.check_status()
        return self._b.statevector(0)

    def amplitude(self, bits: Union[str, Sequence[int]]) -> complex:
        """<b|psi> including exp(norm_log).  A string is read Qiskit-style (last char = qubit 0)."""
        if isinstance(bits, str):
            bits = [int(ch) for ch in reversed(bits)]
        self.check_status()
        return complex(self._b.amplitudes(0, np.asarray(bits)[None, :])[0])

    # -- canonical forms (mps_core.py:219-261) ----------------------------------
    def left_normalize_site(self, i: int) -> None:
        """QR of site i; Q stays, R is absorbed into site i+1 (mps_core.py:221-235)."""
        self._b.canonicalize([0], i, i, "left")

    def right_normalize_site(self, i: int) -> None:
        """LQ of site i; L is absorbed into site i-1 (mps_core.py:237-252)."""
        self._b.canonicalize([0], i, i, "right")

    def left_canonicalize(self) -> None:
        """left_normalize_site(i) for i = 0 .. n-2 (mps_core.py:254-257), one launch."""
        self._b.canonicalize([0], 0, self.n - 2, "left")

    def right_canonicalize(self) -> None:
        """right_normalize_site(i) for i = n-1 .. 1 (mps_core.py:259-261), one launch."""
        self._b.canonicalize([0], 1, self.n - 1, "right")

    def schmidt_values(self, bond: int) -> np.ndarray:
        """Normalised Schmidt coefficients across the cut between sites bond and bond+1.

        The reference reads spectra off its non-canonical gauge
        (``entanglement_entropy`` assumes a mixed-canonical state,
        ``bond_spectrum`` returns the singular values of an isometry, i.e.
        ones); this brings a copy into mixed-canonical form around the cut
        (sites left of it left-normalised, right of it right-normalised) and
        takes the spectrum of the two-site theta there with the fused
        update kernel.  The state itself is not changed.
        """
        if not 0 <= bond < self.n - 1:
            raise ValueError(f"bond {bond} out of range [0, {self.n - 2}]")
        self.check_status()
        m = self.copy()
        m._b.precision = "fp64"
        if bond >= 1:
            m._b.canonicalize([0], 0, bond - 1, "left")
        if bond + 2 <= self.n - 1:
            m._b.canonicalize([0], bond + 2, self.n - 1, "right")
        pb = m._b.apply_layer([0], [bond], np.eye(4, dtype=np.complex128)[None], record_spectra=True)
        s = pb.spectra[0].cpu().numpy()
        s = s[s > 0.0]
        s = s / np.linalg.norm(s)
        return s[s > 1e-15]

    def exact_entanglement_entropy(self, bond: int) -> float:
        """von Neumann entropy -sum p log p of the true Schmidt coefficients at the cut
        after site ``bond`` (``schmidt_values``): exact in any gauge.  The reference's
        ``entanglement_entropy`` equals it only in mixed-canonical form."""
        p = self.schmidt_values(bond) ** 2
        return -float(np.sum(p * np.log(np.maximum(p, 1e-300))))

    def _site_matrix_spectrum(self, m: "MPSState", k: int) -> np.ndarray:
        """Singular values of site k of the scratch copy m read as a (2 chi_l) x chi_r
        matrix, by the fused update kernel: site k+1 is replaced by a row isometry E
        (chi_r x 2 chi', E[b, t, c] = 1 where t chi' + c = b, chi' = ceil(chi_r / 2)),
        so theta = M E has M's singular values, padded with zeros, which the kernel
        records before truncating.  m is consumed."""
        b = m._b
        bonds = b.bonds[: self.n + 1].cpu().numpy()
        cl, cr = int(bonds[k]), int(bonds[k + 1])
        if k == self.n - 1:  # a column: its one singular value is its 2-norm
            return np.array([float(torch.linalg.vector_norm(b.sites[k, : 2 * cl]).item())])
        cp = (cr + 1) // 2
        eye = torch.zeros(b.slot, dtype=torch.complex128, device=b.device)
        rows = torch.arange(cr, device=b.device)
        eye[rows * (2 * cp) + (rows // cp) * cp + rows % cp] = 1.0  # E[b, b // cp, b % cp] = 1
        b.sites[k + 1].copy_(eye)
        b.bonds[k + 2] = cp
        pb = b.apply_layer([0], [k], np.eye(4, dtype=np.complex128)[None], precision="fp64",
                           record_spectra=True)
        s = pb.spectra[0].cpu().numpy()
        return s[: min(2 * cl, cr)]

    def bond_spectrum(self, bond: int) -> np.ndarray:
        """Singular values at ``bond`` as mps_core.py:485-494 computes them: on a copy,
        left-normalise sites 0..bond (QR), then the singular values of site ``bond``
        as a (2 chi_l) x chi_r matrix -- an isometry after the QR, so ones up to
        rounding (``schmidt_values`` gives the Schmidt coefficients)."""
        if not 0 <= bond < self.n:
            raise ValueError(f"bond {bond} out of range [0, {self.n - 1}]")
        self.check_status()
        m = self.copy()
        m._b.canonicalize([0], 0, bond, "left")
        return self._site_matrix_spectrum(m, bond)

    def entanglement_entropy(self, bond: int) -> float:
        """-sum p log p at the bond between sites ``bond`` and ``bond+1`` as
        mps_core.py:465-483 computes it: p = S^2 / sum S^2 over the singular values
        S > 1e-15 of the left block (sites 0..bond contracted into a
        2^(bond+1) x chi matrix).  That is the true entropy only in mixed-canonical
        form; ``exact_entanglement_entropy`` is exact in any gauge.  The left block
        is never formed: after left-normalising sites 0..bond-1 of a copy it equals
        an isometry times site ``bond``, whose singular values the update kernel takes."""
        if not 0 <= bond < self.n - 1:
            raise ValueError(f"bond {bond} out of range [0, {self.n - 2}]")
        self.check_status()
        m = self.copy()
        if bond >= 1:
            m._b.canonicalize([0], 0, bond - 1, "left")
        s = self._site_matrix_spectrum(m, bond)
        s = s[s > 1e-15]
        p = s * s
        p = p / p.sum()
        return -float(np.sum(p * np.log(np.maximum(p, 1e-300))))

    # -- measurement (mps_core.py:354-429) ------------------------------------
    def sample(self, num_shots: int = 1, measured_qubits: Optional[Sequence[int]] = None,
               rng: Optional[np.random.Generator] = None) -> List[str]:
        """Shots as bitstrings (msb = qubit n-1), as MPSState.sample (mps_core.py:371-419).

        The draws use one uniform of ``rng`` per (shot, site), in the order the
        reference's per-site ``rng.choice(2, p=...)`` consumes them, so the
        same seeded generator gives the reference's shots.  For a qubit subset
        the bitstring is bits[n-1-q] over the qubits in decreasing order, as
        the reference builds it (mps_core.py:414-416).
        """
        if rng is None:
            rng = np.random.default_rng()
        if num_shots < 0:
            raise ValueError("num_shots must be >= 0")
        self.check_status()
        u = rng.random((num_shots, self.n))
        bits = self._b.sample_bits(0, u)
        out = []
        subset = measured_qubits is not None and set(measured_qubits) != set(range(self.n))
        ms = sorted(measured_qubits, reverse=True) if subset else None
        chars = np.where(bits == 1, "1", "0")
        for row in chars:
            if subset:
                out.append("".join(row[self.n - 1 - q] for q in ms))
            else:
                out.append("".join(row[::-1]))
        return out

    def get_counts(self, num_shots: int, measured_qubits: Optional[Sequence[int]] = None,
                   rng: Optional[np.random.Generator] = None) -> Dict[str, int]:
        """Sample and count (mps_core.py:421-429)."""
        counts: Dict[str, int] = {}
        for s in self.sample(num_shots, measured_qubits, rng):
            counts[s] = counts.get(s, 0) + 1
        return counts

    def reset(self, site: int) -> None:
        """Site reset of the reference's execution engine (fpga_mps_simulator.py:530-552)."""
        if not 0 <= site < self.n:
            raise ValueError("site out of range")
        self._b.reset_many([0], [site])

    def expectation(self, op: Union[str, Dict[int, np.ndarray]]) -> float:
        """Normalised <psi|O|psi>/<psi|psi> for a local operator.

        ``op`` is a Pauli string in Qiskit order (character k from the left
        acts on qubit n-1-k, as _pauli_expectation_sv reads it,
        fpga_mps_simulator.py:1091-1108) or a dict {site: 2x2 matrix}; the
        non-identity part must sit on one site or two adjacent sites.
        """
        if isinstance(op, str):
            if len(op) != self.n:
                raise ValueError("Pauli string length must equal n")
            op = {self.n - 1 - k: _PAULI[ch.upper()] for k, ch in enumerate(op) if ch.upper() != "I"}
        if not op:
            return 1.0
        ks = sorted(op)
        if len(ks) > 2 or (len(ks) == 2 and ks[1] != ks[0] + 1):
            raise ValueError("expectation supports one site or two adjacent sites")
        self.check_status()
        term = (ks[0], op[ks[0]], op[ks[1]] if len(ks) == 2 else None)
        return float(self._b.expect_terms([term])[0, 0])

    def expect_z_all(self) -> np.ndarray:
        return self._b.expect_terms([(k, _PAULI["Z"], None) for k in range(self.n)])[0]

    def expect_terms(self, terms) -> np.ndarray:
        return self._b.expect_terms(terms)[0]
