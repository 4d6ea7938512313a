"""CPU baseline runner -- TEST/BENCH INFRASTRUCTURE ONLY.

Times the oracle restatement of the reference engine (mps_core.py semantics,
scipy gesdd SVD) on the host cores: one worker process per core, each pinned
to one BLAS thread and advancing its own independent replica of the circuit,
which is how the reference's per-update Python/LAPACK code parallelises
across a CPU.  Workers are started with the "spawn" method so that no forked
child inherits a CUDA context.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os
import time
from typing import Dict, List, Tuple

import numpy as np


def _haar(rng):
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r)
    return q * (d / np.abs(d))[None, :]


def _circuit(n: int, depth: int, seed: int) -> List[Tuple[int, np.ndarray]]:
    rng = np.random.default_rng(seed)
    out = []
    for layer in range(depth):
        for i in range(layer % 2, n - 1, 2):
            out.append((i, _haar(rng)))
    return out


def _worker(args) -> tuple:
    """(updates, seconds) -- plus the final sites and norm_log when `keep` is set,
    so the run can serve as the FP64 reference the device states are checked
    against."""
    n, depth, chi, cutoff, seed, reps, keep = args
    try:
        from threadpoolctl import threadpool_limits
        limiter = threadpool_limits(1)
    except Exception:  # pragma: no cover
        limiter = None
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if here not in sys.path:
        sys.path.insert(0, here)
    from oracle.mps_oracle import OracleMPS
    if limiter is not None:  # again, now that scipy's BLAS is loaded too
        limiter = threadpool_limits(1)
    gates = _circuit(n, depth, seed)
    t0 = time.perf_counter()
    count = 0
    for _ in range(reps):
        st = OracleMPS(n, chi, cutoff, record=False)
        for i, g in gates:
            st.apply_adjacent_2q(i, g)
        count += len(gates)
    dt = time.perf_counter() - t0
    del limiter
    if keep:
        return count, dt, [np.ascontiguousarray(a) for a in st.sites], float(st.norm_log)
    return count, dt


def usable_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def run_parallel(n: int, depth: int, chi: int, cutoff: float, workers: int, reps: int = 1,
                 seed: int = 0, pool=None, keep_first: bool = False) -> Dict[str, float]:
    """Aggregate updates/s of `workers` single-threaded processes, each running `reps` circuits.

    keep_first: also return worker 0's final state (the circuit of `seed`) as
    `final_sites` / `final_norm_log`."""
    own = pool is None
    if own:
        pool = _single_thread_pool(workers)
    try:
        t0 = time.perf_counter()
        res = pool.map(_worker, [(n, depth, chi, cutoff, seed + w, reps, keep_first and w == 0)
                                 for w in range(workers)])
        wall = time.perf_counter() - t0
    finally:
        if own:
            pool.close()
            pool.join()
    updates = sum(r[0] for r in res)
    out = {"updates": updates, "wall_s": wall, "updates_per_s": updates / wall,
           "per_worker_s": float(np.mean([r[1] for r in res])), "workers": workers}
    if keep_first:
        out["final_sites"], out["final_norm_log"] = res[0][2], res[0][3]
    return out


_SINGLE_THREAD_ENV = ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS", "BLIS_NUM_THREADS")


def _single_thread_pool(workers: int):
    """Spawn pool whose workers start with every BLAS thread pool at one thread.
    The variables are read when each BLAS library loads, whatever order a
    worker imports numpy and scipy in; the runtime limit inside the workers
    reaches only libraries already loaded, and scipy's own OpenBLAS loading
    after it left 8 workers x 8 spinning threads on an 8-core host.  The
    parent's environment is restored once the workers exist."""
    saved = {k: os.environ.get(k) for k in _SINGLE_THREAD_ENV}
    try:
        for k in _SINGLE_THREAD_ENV:
            os.environ[k] = "1"
        return mp.get_context("spawn").Pool(workers)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def make_pool(workers: int):
    return _single_thread_pool(workers)


def _grad_worker(args) -> Tuple[int, float]:
    n, layers, chi, cutoff, seed = args
    try:
        from threadpoolctl import threadpool_limits
        limiter = threadpool_limits(1)
    except Exception:  # pragma: no cover
        limiter = None
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if here not in sys.path:
        sys.path.insert(0, here)
    from oracle.mps_adjoint import hea_energy_grad, tfim_mpo
    if limiter is not None:  # again, now that scipy's BLAS is loaded too
        limiter = threadpool_limits(1)
    rng = np.random.default_rng(seed)
    angles = rng.uniform(0.0, 2.0 * math.pi, size=(layers, n, 2))
    t0 = time.perf_counter()
    hea_energy_grad(angles, tfim_mpo(n), chi, cutoff)
    dt = time.perf_counter() - t0
    del limiter
    return 1, dt


def run_grad_parallel(n: int, layers: int, chi: int, cutoff: float, workers: int, seed: int = 0,
                      pool=None) -> Dict[str, float]:
    """Energy + adjoint gradient of one ansatz parameter vector per worker process
    (single BLAS thread each); returns aggregate parameter vectors per second."""
    own = pool is None
    if own:
        pool = _single_thread_pool(workers)
    try:
        t0 = time.perf_counter()
        res = pool.map(_grad_worker, [(n, layers, chi, cutoff, seed + w) for w in range(workers)])
        wall = time.perf_counter() - t0
    finally:
        if own:
            pool.close()
            pool.join()
    vecs = sum(r[0] for r in res)
    return {"vectors": vecs, "wall_s": wall, "vectors_per_s": vecs / wall,
            "per_worker_s": float(np.mean([r[1] for r in res])), "workers": workers}


def _fwd_worker(args) -> Tuple[int, float]:
    n, layers, chi, cutoff, seed = args
    try:
        from threadpoolctl import threadpool_limits
        limiter = threadpool_limits(1)
    except Exception:  # pragma: no cover
        limiter = None
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if here not in sys.path:
        sys.path.insert(0, here)
    from oracle.mps_adjoint import hea_energy, tfim_mpo
    if limiter is not None:  # again, now that scipy's BLAS is loaded too
        limiter = threadpool_limits(1)
    rng = np.random.default_rng(seed)
    angles = rng.uniform(0.0, 2.0 * math.pi, size=(layers, n, 2))
    t0 = time.perf_counter()
    hea_energy(angles, tfim_mpo(n), chi, cutoff)
    dt = time.perf_counter() - t0
    del limiter
    return 1, dt


def run_forward_parallel(n: int, layers: int, chi: int, cutoff: float, workers: int, seed: int = 0,
                         pool=None) -> Dict[str, float]:
    """One ansatz energy evaluation (forward only, the unit of a parameter-shift
    gradient) per worker process; returns the mean seconds per evaluation."""
    own = pool is None
    if own:
        pool = _single_thread_pool(workers)
    try:
        res = pool.map(_fwd_worker, [(n, layers, chi, cutoff, seed + w) for w in range(workers)])
    finally:
        if own:
            pool.close()
            pool.join()
    return {"s_per_eval": float(np.mean([r[1] for r in res])), "workers": workers}


def _default_threads_worker(args) -> Tuple[int, float]:
    chi, count, seed = args
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if here not in sys.path:
        sys.path.insert(0, here)
    from oracle.mps_oracle import OracleMPS
    rng = np.random.default_rng(seed)
    st = OracleMPS(4, chi, 1e-10, record=False)
    for k, (l, r) in enumerate([(1, chi), (chi, chi), (chi, chi), (chi, 1)]):
        st.sites[k] = rng.standard_normal((l, 2, r)) + 1j * rng.standard_normal((l, 2, r))
    gates = [_haar(rng) for _ in range(count)]
    t0 = time.perf_counter()
    for g in gates:
        st.apply_adjacent_2q(1, g)  # a saturated chi x chi x chi update every time
    return count, time.perf_counter() - t0


def single_process_default_threads(chi: int = 64, count: int = 40, seed: int = 0) -> Dict[str, float]:
    """Saturated two-site updates in one process with the BLAS library's default
    thread count (the reference run as-is), in a spawned child."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        k, dt = pool.map(_default_threads_worker, [(chi, count, seed)])[0]
    return {"updates": k, "seconds": dt, "updates_per_s": k / dt}
