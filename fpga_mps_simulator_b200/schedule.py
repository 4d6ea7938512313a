"""Layer schedules for many independent chains, launch strategies, an
autotuner that picks among them, and CUDA-graph capture.

A *schedule* is the sequence of global layers of an ``MPSBatch``: layer L
holds, for every chain that still has a layer L, that chain's disjoint pairs
and gates.  Each layer is one or more launches of the fused update kernel.

Strategies (per layer):

* ``"single"``  -- one launch with the chains in their natural order;
* ``"lpt"``     -- one launch with the chains ordered by decreasing cost
  (largest bond cap first: longest-processing-time-first list scheduling of
  the CTA clusters onto the SMs); each chain's pairs stay contiguous, as the
  norm_log fold requires;
* ``"split"``   -- one launch per bond-cap class, each sized for its own cap
  (fewer rows per lane and less shared memory, so more clusters per SM for
  small chi), on concurrent streams joined at the end of the layer.

and over the whole run:

* ``"flow"``    -- ONE dataflow launch per bond-cap class for all layers
  (``MPSBatch.run_flow``): clusters claim the updates in layer order and each
  starts as soon as the two updates it depends on have finished, so no
  layer waits for the slowest pair of the one before; the classes run on
  concurrent streams joined once, at the end.

``autotune`` times every strategy on the real workload (a window of layers,
on a snapshot of the state that is restored afterwards) and caches the
fastest per workload signature; for ``"flow"`` it first picks, per class,
the CTA size (threads per cluster CTA, from ``_lib.FLOW_THREADS``) that runs
that class's window fastest.  ``Runner.capture`` records a whole schedule in
one CUDA graph for replay.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .circuits import Layer
from .mps import FlowBatch, MPSBatch, PairBatch, _Workspace

__all__ = ["Schedule", "Runner", "autotune", "STRATEGIES", "last_timings", "last_shapes"]

STRATEGIES = ("single", "lpt", "split", "flow")
_TUNE_CACHE: Dict[Tuple, Tuple[str, Dict[int, int]]] = {}
last_timings: Dict[str, float] = {}
last_shapes: Dict[str, Dict[int, float]] = {}


def _cost(chi: int) -> float:
    """Relative cost of one update at bond cap chi (the Jacobi SVD is ~ (2 chi)^3)."""
    return float(chi) ** 3


@dataclass
class _Launch:
    pb: PairBatch
    chi_cap: int


@dataclass
class _FlowLaunch:
    fb: FlowBatch
    chi_cap: int


@dataclass
class Schedule:
    """Per-chain layer lists -> global layers of pair tables for each strategy."""
    batch: MPSBatch
    per_chain: Sequence[Sequence[Layer]]
    record_spectra: bool = False
    _built: Dict[str, List[List[_Launch]]] = field(default_factory=dict)
    flow_threads: Dict[int, int] = field(default_factory=dict)  # cap -> CTA threads of the flow strategy
    _flows: Dict[Tuple[int, int], List[_FlowLaunch]] = field(default_factory=dict)

    def caps(self) -> List[int]:
        """Bond-cap classes, largest first."""
        return sorted(set(self.batch.caps), reverse=True)

    def flow_plan(self, lo: int = 0, hi: Optional[int] = None) -> List[_FlowLaunch]:
        """One work list per bond-cap class covering layers [lo, hi): a chain's
        updates in layer order, within a layer in the layer's own pair order
        (the order the per-layer strategies fold norm_log in)."""
        hi = self.depth if hi is None else min(hi, self.depth)
        key = (lo, hi)
        if key in self._flows:
            return self._flows[key]
        b = self.batch
        out: List[_FlowLaunch] = []
        for cap in self.caps():
            members = [c for c in range(b.nchains) if b.caps[c] == cap]
            ci, si, gs = [], [], []
            for L in range(lo, hi):
                c2, s2, g2 = self._layer_chains(L, members)
                ci += c2
                si += s2
                gs += g2
            if ci:
                out.append(_FlowLaunch(b.make_flow(ci, si, np.concatenate(gs), self.record_spectra), cap))
        self._flows[key] = out
        return out

    @property
    def depth(self) -> int:
        return max((len(ls) for ls in self.per_chain), default=0)

    def updates(self) -> int:
        return sum(len(L.sites) for ls in self.per_chain for L in ls)

    def signature(self) -> Tuple:
        chis = np.asarray(self.batch.caps)
        vals, counts = np.unique(chis, return_counts=True)
        hist = tuple((int(v), int(c)) for v, c in zip(vals, counts))
        return (hist, self.batch.nchains, self.depth, self.updates(), self.batch.precision)

    def _layer_chains(self, L: int, order: Sequence[int]) -> Tuple[list, list, list]:
        ci, si, gs = [], [], []
        for c in order:
            layers = self.per_chain[c]
            if L < len(layers) and len(layers[L].sites):
                ci += [c] * len(layers[L].sites)
                si += [int(i) for i in layers[L].sites]
                gs.append(np.asarray(layers[L].gates))
        return ci, si, gs

    def launches(self, strategy: str) -> List[List[_Launch]]:
        if strategy in self._built:
            return self._built[strategy]
        if strategy not in STRATEGIES:
            raise ValueError(f"unknown strategy {strategy!r}; choose from {STRATEGIES}")
        b = self.batch
        natural = list(range(b.nchains))
        by_cost = sorted(natural, key=lambda c: -_cost(b.caps[c]))
        out: List[List[_Launch]] = []
        for L in range(self.depth):
            ls: List[_Launch] = []
            if strategy in ("single", "lpt"):
                ci, si, gs = self._layer_chains(L, natural if strategy == "single" else by_cost)
                if ci:
                    ls.append(_Launch(b.make_pairs(ci, si, np.concatenate(gs), self.record_spectra),
                                      max(b.caps[c] for c in set(ci))))
            else:
                for cap in sorted(set(b.caps), reverse=True):
                    ci, si, gs = self._layer_chains(L, [c for c in natural if b.caps[c] == cap])
                    if ci:
                        ls.append(_Launch(b.make_pairs(ci, si, np.concatenate(gs), self.record_spectra), cap))
            out.append(ls)
        self._built[strategy] = out
        return out


class Runner:
    """Executes a schedule with one strategy; optionally as one CUDA graph."""

    def __init__(self, schedule: Schedule, strategy: str = "lpt"):
        if strategy not in STRATEGIES:
            raise ValueError(f"unknown strategy {strategy!r}; choose from {STRATEGIES}")
        self.schedule = schedule
        self.strategy = strategy
        self.batch = schedule.batch
        dev = self.batch.device
        self._graph: Optional[torch.cuda.CUDAGraph] = None
        if strategy == "flow":
            n_side = len(schedule.caps())
        else:
            n_side = max((len(ls) for ls in schedule.launches(strategy)), default=1)
        self._streams = [torch.cuda.Stream(dev) for _ in range(n_side)]
        self._ws = [_Workspace(dev) for _ in range(max(n_side, 1))]

    def launches_per_run(self) -> int:
        """Kernel launches of one run (the update kernel and its norm_log fold per launch)."""
        if self.strategy == "flow":
            return 2 * len(self.schedule.flow_plan())
        return 2 * sum(len(ls) for ls in self.schedule.launches(self.strategy))

    def _run_flow(self, lo: int, hi: Optional[int], only_cap: Optional[int] = None,
                  threads: Optional[int] = None) -> None:
        b = self.batch
        sch = self.schedule
        plan = [fl for fl in sch.flow_plan(lo, hi) if only_cap is None or fl.chi_cap == only_cap]

        def go(k, fl, stream=None):
            nt = sch.flow_threads.get(fl.chi_cap, 0) if threads is None else threads
            b.run_flow(fl.fb, chi_cap=fl.chi_cap, threads=nt, workspace=self._ws[k], stream=stream)

        if len(plan) == 1:
            go(0, plan[0])
            return
        main = torch.cuda.current_stream(b.device)
        start = torch.cuda.Event()
        start.record(main)
        ends = []
        for k, fl in enumerate(plan):
            st = self._streams[k]
            st.wait_event(start)
            go(k, fl, st)
            e = torch.cuda.Event()
            e.record(st)
            ends.append(e)
        for e in ends:
            main.wait_event(e)

    def _run_layers(self, lo: int = 0, hi: Optional[int] = None) -> None:
        if self.strategy == "flow":
            self._run_flow(lo, hi)
            return
        b = self.batch
        main = torch.cuda.current_stream(b.device)
        plan = self.schedule.launches(self.strategy)
        for ls in plan[lo: (len(plan) if hi is None else hi)]:
            if len(ls) == 1:
                b.run_pairs(ls[0].pb, chi_cap=ls[0].chi_cap, workspace=self._ws[0])
                continue
            start = torch.cuda.Event()
            start.record(main)
            ends = []
            for k, lc in enumerate(ls):
                st = self._streams[k]
                st.wait_event(start)
                b.run_pairs(lc.pb, chi_cap=lc.chi_cap, workspace=self._ws[k], stream=st)
                e = torch.cuda.Event()
                e.record(st)
                ends.append(e)
            for e in ends:
                main.wait_event(e)

    def run(self, lo: int = 0, hi: Optional[int] = None) -> None:
        """Run layers [lo, hi) eagerly, or the whole schedule by graph replay once captured."""
        if self._graph is not None and lo == 0 and hi is None:
            self._graph.replay()
        else:
            self._run_layers(lo, hi)

    def capture(self) -> None:
        """Record the whole schedule in one CUDA graph.

        One eager run first sizes the workspaces and configures the kernels'
        shared-memory limits, so nothing is allocated or configured inside the
        capture; the state is restored after both runs.
        """
        snap = self.batch.snapshot()
        self._run_layers()
        torch.cuda.synchronize(self.batch.device)
        self.batch.restore(snap)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._run_layers()
        torch.cuda.synchronize(self.batch.device)
        self.batch.restore(snap)
        self._graph = g

    def release(self) -> None:
        self._graph = None


def autotune(schedule: Schedule, start: int = 0, layers: int = 4, repeats: int = 2,
             verbose: bool = False) -> str:
    """Pick the fastest strategy for this schedule (cached per workload signature).

    Every strategy is timed (CUDA events, best of ``repeats``) on layers
    [start, start + layers) from the state the first ``start`` layers leave;
    the batch's state is restored afterwards.
    """
    key = (schedule.signature(), start, layers)
    if key in _TUNE_CACHE:
        best, shapes = _TUNE_CACHE[key]
        schedule.flow_threads.update(shapes)
        return best
    b = schedule.batch
    orig = b.snapshot()
    start = min(start, max(schedule.depth - 1, 0))
    hi = min(start + layers, schedule.depth)
    if start:
        Runner(schedule, "lpt").run(0, start)
    snap = b.snapshot() if start else orig

    def best_of(fn) -> float:
        fn()  # warm-up: first launches configure kernels and size workspaces
        torch.cuda.synchronize(b.device)
        b.restore(snap)
        t = float("inf")
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(b.device)
            t = min(t, e0.elapsed_time(e1))
            b.restore(snap)
        return t

    # CTA shape of the dataflow launch, per bond-cap class (classes are
    # independent chains, so each is timed alone on the window)
    shapes: Dict[int, int] = {}
    shape_ms: Dict[str, Dict[int, float]] = {}
    rflow = Runner(schedule, "flow")
    for cap in schedule.caps():
        menu = _lib.FLOW_THREADS[_lib.rows_per_lane(cap)]
        if b.precision == "mixed_all" or (b.precision in ("mixed", "tf32x3") and _lib.rows_per_lane(cap) == 4):
            menu = menu[:1]  # the tensor-core forms are built for the default CTA size only
        ms = {nt: best_of(lambda: rflow._run_flow(start, hi, only_cap=cap, threads=nt)) for nt in menu}
        shapes[cap] = min(ms, key=ms.get)
        shape_ms[f"chi{cap}"] = {nt: round(v, 3) for nt, v in ms.items()}
    schedule.flow_threads.update(shapes)

    best, best_t = "single", float("inf")
    timings = {}
    for strategy in STRATEGIES:
        r = rflow if strategy == "flow" else Runner(schedule, strategy)
        t = best_of(lambda: r.run(start, hi))
        timings[strategy] = t
        if t < best_t:
            best, best_t = strategy, t
    b.restore(orig)
    if verbose:
        print("autotune", timings, shape_ms, "->", best)
    _TUNE_CACHE[key] = (best, dict(shapes))
    last_timings.clear()
    last_timings.update(timings)
    last_shapes.clear()
    last_shapes.update(shape_ms)
    return best
