"""Circuit lowering, routing, fusion and batched execution on device-resident chains.

``compile_circuit`` mirrors the reference compiler (fpga_mps_simulator.py:285-410):
a circuit -- anything with Qiskit's ``data`` / ``qubits`` / ``num_qubits``
shape, e.g. :class:`Circuit` below or a ``qiskit.QuantumCircuit`` -- becomes
a list of gate dicts on physical sites, every two-site gate on an adjacent
pair.  A permutation ``perm[logical] = physical`` follows the SWAPs; a
non-adjacent pair is routed by SWAPping the far qubit next to the near one,
applying the gate (re-indexed with [0, 2, 1, 3] when the first qubit sits
right of the second) and SWAPping back; ``ccx`` is decomposed into the
standard 15-gate Clifford+T network (whose adjacent CNOTs the reference
places on (min, max) without that re-indexing -- mirrored, so a Toffoli whose
decomposition has a reversed adjacent CNOT reproduces the reference's
result, not the textbook unitary); ``measure`` records physical sites;
``barrier``/``snapshot``/``delay``/``id`` are dropped; ``reset`` is kept.

``schedule`` then packs the gate list into layers for the GPU: single-site
gates on a site are multiplied together and folded into the next two-site
gate that touches the site (the reference applies pending single-site gates
just before each two-site gate, so the result is the same up to rounding);
every remaining operation goes to the earliest layer after the last one
touching its sites.  A layer is at most three launches (single-site gates,
resets, two-site updates).

``MPSSimulator.run`` is the counterpart of ``FPGAMPSSimulator.run``
(fpga_mps_simulator.py:981-1050): several circuits run as independent chains
of one batch, layer by layer, then each is sampled with
``default_rng(seed + index)`` on its measured qubits; :class:`MPSResult`
mirrors ``FPGAMPSResult`` (fpga_mps_simulator.py:733-775).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .gates import GATE_MATRICES, SINGLE_QUBIT_GATES, TWO_QUBIT_GATES, gate_1q, gate_2q, permute_2q
from .mps import MPSBatch, MPSState

__all__ = ["Circuit", "compile_circuit", "schedule", "Program", "MPSSimulator", "MPSResult"]

_ONE_QUBIT = SINGLE_QUBIT_GATES - {"id"}
_TWO_QUBIT = TWO_QUBIT_GATES
_DROPPED = {"barrier", "snapshot", "delay", "id"}
_SWAP = GATE_MATRICES["swap"]


# ----------------------------------------------------------------- circuit builder
class _Qubit:
    __slots__ = ("index",)

    def __init__(self, index: int):
        self.index = index


@dataclass
class _Operation:
    name: str
    params: list


@dataclass
class _Instruction:
    operation: _Operation
    qubits: list


class Circuit:
    """Minimal circuit with the attribute shape of qiskit's QuantumCircuit
    (``num_qubits``, ``qubits``, ``data`` of instructions with ``operation.name``,
    ``operation.params`` and ``qubits``), so the same object feeds this
    compiler and the reference's."""

    def __init__(self, num_qubits: int):
        self.num_qubits = int(num_qubits)
        self.qubits = [_Qubit(i) for i in range(self.num_qubits)]
        self.data: List[_Instruction] = []

    def find_bit(self, q):
        class _Loc:
            def __init__(self, index):
                self.index = index
        return _Loc(q.index)

    def append(self, name: str, qubits: Sequence[int], params: Optional[Sequence[float]] = None) -> "Circuit":
        for q in qubits:
            if not 0 <= q < self.num_qubits:
                raise ValueError(f"qubit {q} out of range")
        self.data.append(_Instruction(_Operation(name, [float(p) for p in (params or [])]),
                                      [self.qubits[q] for q in qubits]))
        return self

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        low = name.lower()
        if low in _ONE_QUBIT or low in ("reset", "measure"):
            return lambda q, *p: self.append(low, [q], p)
        if low in _TWO_QUBIT:
            return lambda a, b, *p: self.append(low, [a, b], p)
        if low in ("ccx", "toffoli", "ccnot"):
            return lambda a, b, c: self.append(low, [a, b, c])
        if low in _DROPPED:
            return lambda *qs: self.append(low, list(qs))
        raise AttributeError(name)

    def measure_all(self) -> "Circuit":
        for q in range(self.num_qubits):
            self.append("measure", [q])
        return self


def _qubit_index(circuit, q) -> int:
    try:
        return circuit.find_bit(q).index
    except Exception:
        return circuit.qubits.index(q)


def _ccx_network(c0: int, c1: int, t: int):
    """Toffoli as H, T, T^dagger and six CNOTs (the textbook 15-gate network)."""
    return [("h", [t]), ("cx", [c1, t]), ("tdg", [t]), ("cx", [c0, t]), ("t", [t]), ("cx", [c1, t]),
            ("tdg", [t]), ("cx", [c0, t]), ("t", [c1]), ("t", [t]), ("h", [t]), ("cx", [c0, c1]),
            ("t", [c0]), ("tdg", [c1]), ("cx", [c0, c1])]


def compile_circuit(circuit, n_qubits: int) -> Tuple[List[dict], List[int]]:
    """Gate list on physical sites and the sorted measured sites (all when none)."""
    perm = list(range(n_qubits))
    out: List[dict] = []
    measured: List[int] = []

    def swap(a: int, b: int) -> None:
        lo, hi = min(a, b), max(a, b)
        out.append({"type": "2q", "gate_name": "swap", "sites": [lo, hi], "params": None, "gate_mat": _SWAP})
        for q in range(n_qubits):
            if perm[q] == lo:
                perm[q] = hi
            elif perm[q] == hi:
                perm[q] = lo

    def two(pi: int, pj: int, name: str, params) -> None:
        g = gate_2q(name, params)
        if abs(pi - pj) == 1:
            if pi > pj:
                out.append({"type": "2q", "gate_name": name, "sites": [pj, pi], "params": params,
                            "gate_mat": permute_2q(g)})
            else:
                out.append({"type": "2q", "gate_name": name, "sites": [pi, pj], "params": params, "gate_mat": g})
            return
        if pi > pj:
            pi, pj = pj, pi
            g = permute_2q(g)
        for k in range(pj, pi + 1, -1):
            swap(k - 1, k)
        out.append({"type": "2q", "gate_name": name, "sites": [pi, pi + 1], "params": params, "gate_mat": g})
        for k in range(pi + 1, pj):
            swap(k, k + 1)

    def one(site: int, name: str, params) -> None:
        out.append({"type": "1q", "gate_name": name, "sites": [site], "params": params,
                    "gate_mat": gate_1q(name, params)})

    for inst in circuit.data:
        name = inst.operation.name.lower()
        qs = [_qubit_index(circuit, q) for q in inst.qubits]
        params = [float(p) for p in getattr(inst.operation, "params", [])] or None
        if name == "measure":
            for q in qs:
                if perm[q] not in measured:
                    measured.append(perm[q])
            continue
        if name in _DROPPED:
            continue
        if name == "reset":
            out.append({"type": "reset", "gate_name": "reset", "sites": [perm[qs[0]]], "params": None,
                        "gate_mat": None})
            continue
        if name in _ONE_QUBIT:
            one(perm[qs[0]], name, params)
            continue
        if name in _TWO_QUBIT:
            two(perm[qs[0]], perm[qs[1]], name, params)
            continue
        if name in ("ccx", "toffoli", "ccnot"):
            for sub, sq in _ccx_network(perm[qs[0]], perm[qs[1]], perm[qs[2]]):
                if len(sq) == 1:
                    one(sq[0], sub, None)
                elif abs(sq[0] - sq[1]) == 1:
                    # as fpga_mps_simulator.py:385-393: an adjacent CNOT of the
                    # decomposition is placed on (min, max) without re-indexing
                    out.append({"type": "2q", "gate_name": sub, "sites": [min(sq), max(sq)], "params": None,
                                "gate_mat": gate_2q(sub, None)})
                else:
                    two(sq[0], sq[1], sub, None)
            continue
        raise ValueError(f"unsupported instruction {name!r}")
    if not measured:
        measured = list(range(n_qubits))
    return out, sorted(measured)


# ----------------------------------------------------------------- scheduling
@dataclass
class Program:
    """Layers of one chain: each layer holds disjoint single-site gates,
    resets and adjacent two-site gates."""
    n: int
    layers: List[dict] = field(default_factory=list)

    @property
    def depth(self) -> int:
        return len(self.layers)

    def counts(self) -> Dict[str, int]:
        return {k: sum(len(L[k]) for L in self.layers) for k in ("one", "reset", "two")}


def schedule(gates: Sequence[dict], n: int, fuse: bool = True) -> Program:
    """Pack a compiled gate list into layers (see module docstring)."""
    pending: Dict[int, np.ndarray] = {}
    layer_of = [0] * n          # first layer free on each site
    layers: List[dict] = []

    def slot(sites: Sequence[int]) -> int:
        L = max(layer_of[s] for s in sites)
        while len(layers) <= L:
            layers.append({"one": [], "reset": [], "two": []})
        for s in sites:
            layer_of[s] = L + 1
        return L

    def flush(site: int) -> None:
        g = pending.pop(site, None)
        if g is not None:
            layers[slot([site])]["one"].append((site, g))

    for op in gates:
        kind, sites = op["type"], op["sites"]
        if kind == "1q":
            s = sites[0]
            g = np.asarray(op["gate_mat"], np.complex128)
            pending[s] = g if s not in pending else g @ pending[s]
            if not fuse:
                flush(s)
        elif kind == "reset":
            flush(sites[0])
            layers[slot(sites)]["reset"].append(sites[0])
        else:
            i, j = sites
            g = np.asarray(op["gate_mat"], np.complex128).reshape(4, 4)
            if fuse:
                gi = pending.pop(i, np.eye(2, dtype=np.complex128))
                gj = pending.pop(j, np.eye(2, dtype=np.complex128))
                g = g @ np.kron(gi, gj)
            else:
                flush(i)
                flush(j)
            layers[slot([i, j])]["two"].append((i, g))
    for s in sorted(pending):
        flush(s)
    return Program(n, layers)


def run_programs(batch: MPSBatch, programs: Sequence[Program]) -> int:
    """Execute one program per chain of ``batch`` (chain c = programs[c]), global
    layer by layer; returns the number of launches."""
    depth = max((p.depth for p in programs), default=0)
    launches = 0
    for L in range(depth):
        c1, s1, g1, cr, sr, c2, s2, g2 = [], [], [], [], [], [], [], []
        for c, p in enumerate(programs):
            if L >= p.depth:
                continue
            lay = p.layers[L]
            for s, g in lay["one"]:
                c1.append(c); s1.append(s); g1.append(g)
            for s in lay["reset"]:
                cr.append(c); sr.append(s)
            for i, g in sorted(lay["two"], key=lambda t: t[0]):
                c2.append(c); s2.append(i); g2.append(g)
        if c1:
            batch.apply_1q_many(c1, s1, np.stack(g1))
            launches += 1
        if cr:
            batch.reset_many(cr, sr)
            launches += 1
        if c2:
            batch.apply_layer(c2, s2, np.stack(g2))
            launches += 2
    return launches


# ----------------------------------------------------------------- simulator
class MPSResult:
    """Result container with the accessors of FPGAMPSResult (fpga_mps_simulator.py:733-775)."""

    def __init__(self, results: list, shots: int, elapsed: float, mode: str = "shots_b200"):
        self._results = results
        self.shots = shots
        self.num_cards = 1
        self.total_time = elapsed
        self.mode = mode

    def get_counts(self, idx: int = 0) -> Dict[str, int]:
        return self._results[idx]["counts"]

    def get_statevector(self, idx: int = 0) -> np.ndarray:
        sv = self._results[idx].get("statevector")
        if sv is None:
            raise ValueError("Statevector not available (n > 24 or not computed).")
        return sv

    def get_mps(self, idx: int = 0) -> Optional[MPSState]:
        return self._results[idx].get("mps")

    def get_max_bond(self, idx: int = 0) -> int:
        return self._results[idx].get("max_bond", -1)

    def get_bond_dims(self, idx: int = 0) -> List[int]:
        return self._results[idx].get("bond_dims", [])

    def get_phase_times(self, idx: int = 0) -> Dict[str, float]:
        return self._results[idx].get("phase_times", {})

    def success(self) -> bool:
        return True


class MPSSimulator:
    """Counterpart of FPGAMPSSimulator (fpga_mps_simulator.py:778-1050) on one B200.

    ``run(circuits, shots, seed)`` compiles every circuit, runs them together
    as independent chains of one device batch (global layers: one launch per
    kind of operation), reads each chain back as an ``MPSState`` and samples
    it with ``default_rng(seed + index)`` (``None`` seed: fresh entropy), as
    the reference does per circuit.
    """

    def __init__(self, chi_max: int = 64, svd_cutoff: float = 1e-12, precision: str = "fp64",
                 device="cuda", fuse_1q: bool = True):
        self.chi_max = int(chi_max)
        self.svd_cutoff = float(svd_cutoff)
        self.precision = precision
        self.device = device
        self.fuse_1q = fuse_1q

    def run(self, circuits, shots: int = 1024, seed: Optional[int] = None) -> MPSResult:
        if not isinstance(circuits, (list, tuple)):
            circuits = [circuits]
        t0 = time.time()
        compiled = []
        for c in circuits:
            gl, meas = compile_circuit(c, c.num_qubits)
            compiled.append((c.num_qubits, schedule(gl, c.num_qubits, self.fuse_1q), meas))
        t_compile = time.time() - t0
        batch = MPSBatch([n for n, _, _ in compiled], self.chi_max, self.svd_cutoff, precision=self.precision,
                         device=self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launches = run_programs(batch, [p for _, p, _ in compiled])
        e1.record()
        torch.cuda.synchronize(batch.device)
        batch.check_status()
        gpu_s = e0.elapsed_time(e1) * 1e-3
        results = []
        for idx, (n, prog, meas) in enumerate(compiled):
            st = MPSState(n, self.chi_max, self.svd_cutoff, self.precision, batch.device)
            o = int(batch.site_off[idx])
            # the chain's bonds fit its own cap, so the head of each batch slot holds the whole site
            st._b.sites[:n].copy_(batch.sites[o:o + n, : st._b.slot])
            b0 = int(batch.bond_off[idx])
            st._b.bonds.copy_(batch.bonds[b0:b0 + n + 1])
            st._b.norm_logs[0] = batch.norm_logs[idx]
            ts = time.time()
            rng = np.random.default_rng(None if seed is None else seed + idx)
            counts = st.get_counts(shots, meas, rng)
            t_sample = time.time() - ts
            sv = st.get_statevector() if n <= 24 else None
            results.append({"counts": counts, "statevector": sv, "mps": st, "max_bond": st.max_bond(),
                            "bond_dims": st.bond_dims(),
                            "phase_times": {"compile": t_compile, "gpu_layers": gpu_s, "sampling": t_sample,
                                            "launches": launches, "layers": prog.depth}})
        return MPSResult(results, shots, time.time() - t0)
