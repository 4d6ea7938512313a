#!/usr/bin/env python
"""Benchmark: MPS two-site updates/s at chi_max = 64 on B200.

Workload (one "step"): a 100-qubit open chain in |0...0>, depth-20 brick-wall
of Haar-random 4x4 gates (seeded), chi_max = 64, cutoff 1e-10 -- 990 two-site
updates, all 20 layers in one dataflow launch (each pair starts when the two
updates before it on its sites are done); one launch per layer (49-50 pairs
each) is timed beside it, with bit-identical results.  Synthetic gates; no
dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value`` is device-timed (CUDA events, inputs resident in HBM, L2 flushed
between steps) updates/s over all ranks; ``e2e`` runs the same circuit
through the public Python API (``MPSState.apply_layers``) with the gates copied
from pinned host memory and the final MPS read back every step.  With
--gpus N > 1 (launched by torch.distributed.run) every rank advances its own
replica circuit (different seed): no collective on the data path, timing is
the max over ranks.  ``--impl reference`` times the CPU restatement of the
reference engine (scipy gesdd) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MPS 2-site updates/s at chi=64 and grad s/step: mixed vs FP64 GPU, err≤1e-6"
UNIT = "updates/s"
N_SITES, DEPTH, CHI, CUTOFF, SEED = 100, 20, 64, 1e-10, 2024
WORKLOAD = (f"MPS two-site updates: n={N_SITES} open chain, depth-{DEPTH} Haar brick-wall, "
            f"chi_max={CHI}, cutoff={CUTOFF:g}; all layers' pairs in one dataflow launch "
            "(per-layer launches reported beside it)")


# DRAM bytes (read + write) of one dataflow launch (the whole 990-update step,
# mixed form), from one ncu capture of this workload: 1.15 MB read + 3.36 MB
# written (sites and theta copies stay in L2).
TRAFFIC_PER_LAUNCH = 5.30e6
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one dataflow launch of this "
                  "workload (990 updates); algorithmic site bytes per step in hbm_site_bytes_per_step")

# ----------------------------------------------------------------- counting
def update_flops(cl: int, cm: int, cr: int) -> float:
    """Algorithmic flops of one update: contraction 32 cl cm cr, gate 128 cl cr,
    nominal complex SVD 4 (14 m n^2 + 8 n^3) with m >= n the sides of theta."""
    m, n = 2 * cl, 2 * cr
    if m < n:
        m, n = n, m
    return 32.0 * cl * cm * cr + 128.0 * cl * cr + 4.0 * (14.0 * m * n * n + 8.0 * n ** 3)


def update_bytes(cl: int, cm: int, cr: int, k: int) -> float:
    """Site-tensor HBM bytes of one update: read A, B and the gate, write A', B'."""
    return 16.0 * (2 * cl * cm + 2 * cm * cr + 2 * cl * k + 2 * k * cr) + 256.0


def replay_dims(n: int, layer_sites, layer_kept):
    """Pre-update (chi_l, chi_m, chi_r, kept) of every pair, replayed from the kept counts."""
    bonds = [1] * (n + 1)
    out = []
    for sites, kept in zip(layer_sites, layer_kept):
        per = []
        for i, k in zip(sites, kept):
            per.append((bonds[i], bonds[i + 1], bonds[i + 2], int(k)))
        for i, k in zip(sites, kept):
            bonds[i + 1] = int(k)
        out.append(per)
    return out


BATCH_CIRCUITS, BATCH_N, BATCH_DEPTH, BATCH_CHIS = 256, (20, 200), (10, 40), (16, 32, 64)


def batching_leg(dev, steps: int, rank: int, max_over_ranks, precision: str = "mixed"):
    """Many uneven circuits: 256 Haar brick-walls, n ~ U[20,200], depth ~ U[10,40],
    chi_max from {16,32,64}, cutoff 1e-10.  The autotuned launch strategy is
    captured in one CUDA graph and replayed (device-timed per full run); the
    comparison is a one-circuit-at-a-time loop of per-layer launches."""
    import torch
    from fpga_mps_simulator_b200 import MPSBatch
    from fpga_mps_simulator_b200.circuits import random_circuit_batch
    from fpga_mps_simulator_b200.schedule import Runner, Schedule, autotune, last_shapes, last_timings

    specs = random_circuit_batch(BATCH_CIRCUITS, seed=SEED + rank, n_range=BATCH_N, depth_range=BATCH_DEPTH,
                                 chis=BATCH_CHIS)
    b = MPSBatch([s.n for s in specs], [s.chi_max for s in specs], CUTOFF, precision=precision, device=dev)
    sch = Schedule(b, [s.layers for s in specs])
    n_upd = sch.updates()
    init = b.snapshot()
    best = autotune(sch, start=12, layers=4, repeats=2)
    tuned = dict(last_timings)
    shapes = {k: dict(v) for k, v in last_shapes.items()}
    flow_threads = {f"chi{k}": v for k, v in sch.flow_threads.items()}
    r = Runner(sch, best)
    r.capture()

    def timed(fn):
        b.restore(init)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    timed(r.run)  # warm replay
    run_s = [timed(r.run) for _ in range(steps)]
    b.check_status()
    graph_s = max_over_ranks(sum(run_s)) / steps
    launches = r.launches_per_run()
    r.release()

    # one circuit at a time: each circuit's layers launched in turn, sized for that circuit
    loop_plan = []
    for c, s in enumerate(specs):
        for L in s.layers:
            loop_plan.append(b.make_pairs(np.full(len(L.sites), c, np.int32), L.sites, L.gates))

    def loop():
        k = 0
        for s in specs:
            for _ in s.layers:
                b.run_pairs(loop_plan[k], chi_cap=s.chi_max)
                k += 1

    loop_s = max_over_ranks(timed(loop))
    b.check_status()
    return {"workload": (f"{BATCH_CIRCUITS} Haar brick-wall circuits, n~U{list(BATCH_N)}, "
                         f"depth~U{list(BATCH_DEPTH)}, chi_max in {list(BATCH_CHIS)}, cutoff {CUTOFF:g}, "
                         f"{precision} form"),
            "updates_per_run": n_upd, "strategy": best, "launches_per_run": launches,
            "autotune_ms": {k: round(v, 3) for k, v in tuned.items()},
            "flow_cta_threads": flow_threads, "flow_shape_ms": shapes,
            "graph_updates_per_s": round(n_upd / graph_s, 3), "graph_s_per_run": round(graph_s, 4),
            "loop_updates_per_s": round(n_upd / loop_s, 3), "loop_s_per_run": round(loop_s, 4),
            "speedup_vs_loop": round(loop_s / graph_s, 3),
            "note": ("graph = whole run captured as one CUDA graph; loop = one launch per circuit layer; "
                     "strategies: single / lpt / split launch per layer, flow = one dataflow launch per "
                     "bond-cap class for all layers (CTA threads per class picked by the autotuner)")}


GRAD_N, GRAD_LAYERS, GRAD_VEC, GRAD_CHI, GRAD_CUT = 64, 8, 64, 32, 1e-12


def _svd_flops(cl: int, cr: int) -> float:
    m, n = 2 * cl, 2 * cr
    if m < n:
        m, n = n, m
    return 4.0 * (14.0 * m * n * n + 8.0 * n ** 3)


def hea_grad_flops(model, angles) -> float:
    """Algorithmic flops of one energy + gradient step: per update the forward
    (contraction, gate, nominal SVD) plus the backward counted as twice the
    contraction and twice the SVD; dims replayed from an untimed forward."""
    import torch
    from fpga_mps_simulator_b200.adjoint import Step2Q
    model._set_angles(angles)
    model._reset()
    b = model.batch
    total = 0.0
    for g in model.groups:
        for st in g:
            if isinstance(st, Step2Q):
                bonds = b.bonds.cpu().numpy()
                pairs = st.pb.pairs.cpu().numpy()
                for c, i in pairs[:, :2]:
                    o = int(b.bond_off[c]) + int(i)
                    cl, cm, cr = int(bonds[o]), int(bonds[o + 1]), int(bonds[o + 2])
                    contr = 32.0 * cl * cm * cr
                    total += 3.0 * contr + 128.0 * cl * cr + 3.0 * _svd_flops(cl, cr)
            model.engine._run(st)
    torch.cuda.synchronize()
    return total


GRAD_CHECK_PARAMS, GRAD_CHECK_H = 20, 1e-4


def gradient_check(dev, n: int, layers: int, chi: int, angles0: np.ndarray, adjoints: dict, seed: int):
    """Adjoint gradients of one parameter vector against the plain (FP64) forward:
    parameter shift (E(x + pi/2) - E(x - pi/2)) / 2 and central differences with
    h = 1e-4 on GRAD_CHECK_PARAMS sampled angles, all 4 x GRAD_CHECK_PARAMS shifted
    vectors run as chains of one batch.  Errors are relative to the largest
    |gradient| of the sample (the scale of the test bar 1e-5)."""
    from fpga_mps_simulator_b200.adjoint import HEAEnergy
    rng = np.random.default_rng(seed)
    flat = rng.choice(layers * n * 2, size=GRAD_CHECK_PARAMS, replace=False)
    picks = [np.unravel_index(int(f), (layers, n, 2)) for f in flat]
    shifts = [math.pi / 2, -math.pi / 2, GRAD_CHECK_H, -GRAD_CHECK_H]
    shifted = np.repeat(angles0[None], len(shifts) * len(picks), 0)
    for p, idx in enumerate(picks):
        for k, d in enumerate(shifts):
            shifted[len(shifts) * p + k][idx] += d
    model = HEAEnergy(n, layers, len(shifted), chi_max=chi, cutoff=GRAD_CUT, precision="fp64", device=dev)
    es = model.forward(shifted).cpu().numpy().reshape(len(picks), len(shifts))
    bonds = max(max(model.batch.bond_dims(c)) for c in range(0, len(shifted), len(shifts)))
    del model
    ps = 0.5 * (es[:, 0] - es[:, 1])
    fd = (es[:, 2] - es[:, 3]) / (2 * GRAD_CHECK_H)
    out = {"params": GRAD_CHECK_PARAMS, "fd_h": GRAD_CHECK_H, "max_bond": int(bonds),
           "max_abs_grad": float(np.max(np.abs(ps)))}
    scale = max(float(np.max(np.abs(ps))), 1e-12)
    for form, g in adjoints.items():
        adj = np.array([g[idx] for idx in picks])
        out[f"{form}_adjoint_vs_parameter_shift"] = float(np.max(np.abs(adj - ps)) / scale)
        out[f"{form}_adjoint_vs_fd"] = float(np.max(np.abs(adj - fd)) / scale)
    out["parameter_shift_vs_fd"] = float(np.max(np.abs(ps - fd)) / scale)
    return out


def gradient_leg(dev, steps: int, warmup: int, rank: int, max_over_ranks, cpu_workers: int = 0):
    """Energy + adjoint gradient of 64 hardware-efficient-ansatz parameter vectors
    (n=64, 8 layers of RY, RZ and brick-wall CZ, chi_max=32, transverse-field
    Ising energy) per step, with per-layer checkpointing; both forms."""
    import torch
    from fpga_mps_simulator_b200.adjoint import HEAEnergy
    from fpga_mps_simulator_b200.circuits import hea_angles
    angles = torch.tensor(hea_angles(GRAD_N, GRAD_LAYERS, GRAD_VEC, SEED + rank), dtype=torch.float64, device=dev)
    out, grads, finals = {}, {}, {}
    flops = None
    for prec, ckpt in (("fp64", "auto"), ("mixed", "auto"), ("mixed_all", "auto"), ("fp64", True)):
        model = HEAEnergy(GRAD_N, GRAD_LAYERS, GRAD_VEC, chi_max=GRAD_CHI, cutoff=GRAD_CUT, precision=prec,
                          device=dev, checkpoint=ckpt)
        for _ in range(warmup):
            model.energy_and_grad(angles)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        base_mem = torch.cuda.memory_allocated(dev)
        model.engine.launches = 0
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        evs[0].record()
        for k in range(steps):
            E, g = model.energy_and_grad(angles)
            evs[k + 1].record()
        torch.cuda.synchronize()
        sec = max_over_ranks(evs[0].elapsed_time(evs[-1]) * 1e-3) / steps
        step_s = [round(evs[k].elapsed_time(evs[k + 1]) * 1e-3, 5) for k in range(steps)]
        key = prec if ckpt == "auto" else f"{prec}_checkpointed"
        grads[key] = (E.clone(), g.clone())
        if ckpt == "auto":
            finals[prec] = model.batch
        if flops is None:
            flops = hea_grad_flops(model, angles)
        out[key] = {"s_per_grad_step": round(sec, 5), "step_s": step_s, "grad_steps_per_s": round(1.0 / sec, 4),
                    "param_vectors_per_s": round(GRAD_VEC / sec, 3),
                    "recompute": bool(model.engine.checkpointed),
                    "launches_per_step": model.engine.launches // steps,
                    "peak_mem_gb": round((torch.cuda.max_memory_allocated(dev) - base_mem) / 1e9, 3),
                    "achieved_tflops": round(flops / sec / 1e12, 4)}
        del model
        torch.cuda.empty_cache()
    from fpga_mps_simulator_b200.mps import overlap

    def versus_fp64(form: str) -> dict:
        infid = []
        for c in range(GRAD_VEC):  # final ansatz states, this form vs FP64
            ab, lab = overlap(finals[form], c, finals["fp64"], c)
            aa, laa = overlap(finals[form], c, finals[form], c)
            bb, lbb = overlap(finals["fp64"], c, finals["fp64"], c)
            infid.append(1.0 - abs(ab) ** 2 / (aa.real * bb.real) * math.exp(2 * lab - laa - lbb))
        (e64, g64), (emx, gmx) = grads["fp64"], grads[form]
        return {"max_abs_energy_diff": float(torch.max(torch.abs(emx - e64))),
                "max_rel_grad_diff": float(torch.max(torch.abs(gmx - g64)) / torch.max(torch.abs(g64))),
                "grad_rel_diff_median": float(torch.median(
                    torch.amax(torch.abs(gmx - g64), dim=(1, 2, 3)) / torch.amax(torch.abs(g64), dim=(1, 2, 3)))),
                "state_infidelity_median": float(np.median(infid)),
                "state_infidelity_max": float(np.max(infid))}

    cmp_mixed, cmp_all = versus_fp64("mixed"), versus_fp64("mixed_all")
    finals.clear()
    res = {"workload": (f"{GRAD_VEC} parameter vectors of a {GRAD_N}-qubit hardware-efficient ansatz, "
                        f"{GRAD_LAYERS} layers (RY, RZ every site, CZ brick-wall), chi_max={GRAD_CHI}, "
                        f"transverse-field Ising energy J=h=1; energy + adjoint gradient per step; "
                        f"tapes kept in HBM (recompute false) or per-layer checkpoints + recomputation"),
           "fp64": out["fp64"], "mixed": out["mixed"], "mixed_all": out["mixed_all"],
           "fp64_checkpointed": out["fp64_checkpointed"],
           "mixed_form_note": ("at chi_cap <= 32 'mixed' runs the exact FP64 contraction and differs from fp64 only "
                               "by its Jacobi tolerance, 1e-9 against 1e-14; 'mixed_all' takes the 3xTF32 "
                               "tensor-core contraction here too (64-row tcgen05 tiles) with the 1e-6 S[0] floor"),
           "checkpointed_equals_taped": bool(torch.equal(grads["fp64"][1], grads["fp64_checkpointed"][1])),
           "mixed_vs_fp64": dict(cmp_mixed, note=(
               "per parameter vector; the largest gradient differences on vectors with near-degenerate singular "
               "values at the truncation boundary")),
           "mixed_all_vs_fp64": dict(cmp_all, note=(
               "the tensor-core theta's ~1e-7 relative rounding and its 1e-6 S[0] floor change which values the "
               "truncation keeps on these graded spectra")),
           "flops_per_step": flops}
    # adjoint vs parameter shift and central differences on the plain forward,
    # at this size (8 layers: bonds reach chi_max = 32 and truncate) and on a
    # 4-layer control of the same chain (bonds <= 2^4 = 16: no chi truncation)
    a0 = angles[0].cpu().numpy()
    check = gradient_check(dev, GRAD_N, GRAD_LAYERS, GRAD_CHI, a0,
                           {"fp64": grads["fp64"][1][0].cpu().numpy(),
                            "mixed": grads["mixed"][1][0].cpu().numpy(),
                            "mixed_all": grads["mixed_all"][1][0].cpu().numpy()}, SEED + 7)
    ctl_layers = 4
    ctl = {}
    for prec in ("fp64", "mixed", "mixed_all"):
        m4 = HEAEnergy(GRAD_N, ctl_layers, 1, chi_max=GRAD_CHI, cutoff=GRAD_CUT, precision=prec, device=dev)
        ctl[prec] = m4.energy_and_grad(a0[None, :ctl_layers])[1][0].cpu().numpy()
        del m4
    control = gradient_check(dev, GRAD_N, ctl_layers, GRAD_CHI, a0[:ctl_layers], ctl, SEED + 8)
    torch.cuda.empty_cache()
    res["gradient_check"] = {
        "config": check, f"control_{ctl_layers}_layers": control,
        "bar": "adjoint within 1e-5 of parameter shift, relative to the largest |gradient|",
        "note": ("parameter shift and central differences run the plain FP64 forward on one parameter vector; "
                 "at 8 layers the bonds saturate at chi_max=32: the truncated energy is no longer a sinusoid "
                 "in each angle, so the parameter-shift rule itself stops being a derivative (compare "
                 "parameter_shift_vs_fd), while central differences still measure the derivative the adjoint "
                 f"computes; the {ctl_layers}-layer control has no chi truncation, where all three agree")}
    if cpu_workers:
        from oracle.cpu_baseline import make_pool, run_forward_parallel, run_grad_parallel
        pool = make_pool(cpu_workers)
        try:
            run_grad_parallel(8, 1, 4, GRAD_CUT, cpu_workers, pool=pool)
            r = run_grad_parallel(GRAD_N, GRAD_LAYERS, GRAD_CHI, GRAD_CUT, cpu_workers, seed=SEED, pool=pool)
            f = run_forward_parallel(GRAD_N, GRAD_LAYERS, GRAD_CHI, GRAD_CUT, cpu_workers, seed=SEED, pool=pool)
        finally:
            pool.close()
            pool.join()
        n_params = GRAD_LAYERS * GRAD_N * 2
        ps_step = (2 * n_params + 1) * f["s_per_eval"] * GRAD_VEC / cpu_workers
        res["cpu_parameter_shift"] = {
            "value": round(ps_step, 1), "unit": "s/grad step", "cores": cpu_workers, "kind": "port",
            "sample": (f"one energy evaluation per process ({f['s_per_eval']:.2f} s, the reference's update "
                       f"semantics), extrapolated to 2P+1 = {2 * n_params + 1} evaluations per vector x "
                       f"{GRAD_VEC} vectors over {cpu_workers} processes: the parameter-shift gradient the "
                       "reference engine would need")}
        res["cpu_baseline"] = {"value": round(GRAD_VEC / r["vectors_per_s"], 3), "unit": "s/grad step",
                               "cores": cpu_workers, "kind": "port",
                               "sample": (f"{cpu_workers} single-BLAS-thread processes, one parameter vector each "
                                          f"({r['wall_s']:.1f} s wall), CPU adjoint oracle (scipy gesdd); "
                                          f"extrapolated to {GRAD_VEC} vectors")}
    return res


LARGE_N, LARGE_STEPS, LARGE_DT, LARGE_CHI, LARGE_CUT, LARGE_FD = 1000, 30, 0.05, 64, 1e-10, 20


def large_leg(dev, precision: str = "fp64"):
    """1000-qubit open XXZ chain (Jxy=1, Jz=0.5), 30 second-order Trotter steps of
    dt=0.05 from a seeded random product state, chi_max=64, cutoff 1e-10: the
    gradient of sum <Z_i Z_{i+1}> with respect to the 2000 initial Bloch angles
    with per-Trotter-step checkpointing, its memory high-water, and central
    differences (h=1e-5) on 20 sampled angles run as one 40-chain forward."""
    import torch
    from fpga_mps_simulator_b200 import MPSBatch
    from fpga_mps_simulator_b200.adjoint import AdjointEngine, XXZInitialStateGradient
    from fpga_mps_simulator_b200.circuits import random_product_angles, xxz_trotter_layers
    from fpga_mps_simulator_b200.hamiltonians import zz_mpo
    angles = random_product_angles(LARGE_N, SEED)
    modes = {}
    for ckpt in (True, False):
        model = XXZInitialStateGradient(LARGE_N, LARGE_STEPS, LARGE_DT, 1.0, 0.5, chi_max=LARGE_CHI,
                                        cutoff=LARGE_CUT, precision=precision, device=dev, checkpoint=ckpt)
        # warm-up: also leaves the tapes' device blocks in the allocator's cache,
        # so the timed call measures the kernels, not a fresh 37 GB allocation
        # (the peak below counts allocated bytes, so the cache does not inflate it)
        model.energy_and_grad(angles)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        base = torch.cuda.memory_allocated(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        energy, grad = model.energy_and_grad(angles)
        e1.record()
        torch.cuda.synchronize()
        key = "checkpointed" if ckpt else "tapes_in_hbm"
        modes[key] = {"s_energy_and_grad": round(e0.elapsed_time(e1) * 1e-3, 4),
                      "peak_mem_gb": round((torch.cuda.max_memory_allocated(dev) - base) / 1e9, 3)}
        if not ckpt:
            break
        del model
    sec = modes["checkpointed"]["s_energy_and_grad"]
    peak = modes["checkpointed"]["peak_mem_gb"] * 1e9
    bonds = model.batch.bond_dims(0)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    e_fwd = model.energy(angles)
    f1.record()
    torch.cuda.synchronize()
    fwd_s = f0.elapsed_time(f1) * 1e-3
    grad = grad.cpu().numpy()
    del model
    torch.cuda.empty_cache()
    # central differences: 2 x 20 perturbed initial states as independent chains of one batch
    rng = np.random.default_rng(SEED + 1)
    flat = rng.choice(LARGE_N * 2, size=LARGE_FD, replace=False)
    picks = [(int(f) // 2, int(f) % 2) for f in flat]
    h = 1e-5
    nch = 2 * LARGE_FD
    b = MPSBatch([LARGE_N] * nch, LARGE_CHI, LARGE_CUT, precision=precision, device=dev)
    th = np.repeat(angles[None], nch, 0)
    for p, idx in enumerate(picks):
        th[2 * p][idx] += h
        th[2 * p + 1][idx] -= h
    t = torch.tensor(th.reshape(-1, 2), dtype=torch.float64, device=dev)
    b.sites.zero_()
    b.sites[:, 0] = torch.cos(0.5 * t[:, 0]).to(torch.complex128)
    b.sites[:, 1] = torch.exp(1j * t[:, 1]) * torch.sin(0.5 * t[:, 0])
    for L in xxz_trotter_layers(LARGE_N, LARGE_STEPS, LARGE_DT, 1.0, 0.5):
        ci = np.repeat(np.arange(nch, dtype=np.int32), len(L.sites))
        si = np.tile(L.sites, nch)
        b.apply_layer(ci, si, np.tile(L.gates, (nch, 1, 1)))
    b.check_status()
    es = AdjointEngine(b, zz_mpo(LARGE_N)).energy().cpu().numpy()
    fd = (es[0::2] - es[1::2]) / (2 * h)
    adj = np.array([grad[idx] for idx in picks])
    err = np.abs(adj - fd)
    del b
    torch.cuda.empty_cache()
    return {"workload": (f"{LARGE_N}-qubit XXZ (Jxy=1, Jz=0.5), {LARGE_STEPS} second-order Trotter steps dt={LARGE_DT}, "
                         f"random product start, chi_max={LARGE_CHI}, cutoff {LARGE_CUT:g}, {precision}; "
                         "d sum<ZZ> / d initial angles, per-Trotter-step checkpointing"),
            "energy": energy, "energy_forward_only": e_fwd, "s_energy_and_grad": round(sec, 4),
            "s_forward_only": round(fwd_s, 4), "peak_mem_gb": round(peak / 1e9, 3), "modes": modes,
            "max_bond": max(bonds),
            "fd_check": {"angles": LARGE_FD, "h": h, "max_abs_err": float(err.max()),
                         "max_rel_err": float((err / np.maximum(np.abs(fd), 1e-12)).max()),
                         "max_abs_grad": float(np.abs(grad).max())}}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples taken while the timed region runs.

    nvidia-smi takes a few hundred ms to produce its first sample and may hold
    its output until it exits, so it is started ahead of the timed region
    (begin() marks the region's start, stop() its end) and every sample
    carries its own timestamp: the samples inside the region are kept, and
    when the region is shorter than the sampling interval, the nearest sample
    on each side of it.
    """

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 50

    def __init__(self, gpu_id: str):
        import datetime
        self._now = datetime.datetime.now
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.t0 = self.t1 = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.8)  # first samples under way before the region starts
        except Exception:
            self.proc = None

    def begin(self) -> None:
        self.t0 = self._now()

    def stop(self):
        import datetime
        if self.proc is None:
            return None
        self.t1 = self._now()
        time.sleep(2.0 * self.PERIOD_MS / 1000.0)  # one more sample after the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm_mhz, max_mhz = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                ts = None
            rows.append((ts, sm_mhz, max_mhz, parts[6:10]))
        os.unlink(self.path)
        t0 = self.t0 or self.t1
        if any(r[0] is None for r in rows):  # unreadable timestamps: every sample counts
            inside = rows
        else:
            inside = [r for r in rows if t0 <= r[0] <= self.t1]
        if not inside and rows and rows[0][0] is not None:  # region shorter than the period: the neighbours
            before = [r for r in rows if r[0] < t0]
            after = [r for r in rows if r[0] > self.t1]
            inside = before[-1:] + after[:1]
        if not inside:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {nm for r in inside for nm, v in zip(names, r[3]) if v.lower().startswith("active")}
        sm = [r[1] for r in inside]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(r[2] for r in inside)),
                "reasons": sorted(reasons), "samples": len(sm),
                "region_s": round((self.t1 - t0).total_seconds(), 3)}


# ----------------------------------------------------------------- CPU side
def contraction_leg(dev, batch, gates, steps: int, fp64_peak_tflops: float, update_s_per_update: float):
    """theta = G (A B) alone (mpsb_contract2q_batch, the FPGA offload's piece), both forms,
    on the finished config-2 state: its 99 adjacent pairs ten times over (990 thetas,
    259 MB of output, larger than L2), device-timed per launch.  The tensor-core form is
    held to a measured tcgen05 TF32 peak, the FP64 form to the FP64 probe."""
    import torch
    from fpga_mps_simulator_b200 import _lib
    lib = _lib.load()
    n = batch.ns[0]
    reps = 10
    sites = np.tile(np.arange(n - 1), reps)
    tb = batch.make_thetas(np.zeros(len(sites), np.int32), sites, gates[: len(sites)])
    bonds = batch.bonds.cpu().numpy()
    dims = [(int(bonds[i]), int(bonds[i + 1]), int(bonds[i + 2])) for i in sites]
    alg = float(sum(32.0 * cl * cm * cr + 128.0 * cl * cr for cl, cm, cr in dims))
    # tensor-core flops the 3xTF32 complex-3M form issues: per CTA (two per pair, each
    # half of the columns) 3 products x 3 MMAs per K = 8 step, M = 128 rows
    issued = 0.0
    for cl, cm, cr in dims:
        w = ((2 * cr + 15) & ~15) >> 2
        for half in (0, 1):
            nidx = max(0, min(cr, half * w + w) - half * w)
            if nidx:
                npad = max(16, (2 * nidx + 15) & ~15)
                issued += 9 * 2.0 * 128 * npad * ((cm + 7) & ~7)
    s = torch.cuda.current_stream(dev)
    res = {"pairs": len(sites), "flops_per_launch": alg, "workload": "config-2 final state, 99 pairs x 10"}
    for form in ("fp64", "mixed"):
        for _ in range(3):
            batch.run_thetas(tb, form)
        torch.cuda.synchronize()
        if tb.status.any().item():
            raise RuntimeError("contraction leg: a pair reported " + str(tb.status.cpu().numpy().max()))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps)]
        for k in range(steps):
            ev[2 * k].record(s)
            batch.run_thetas(tb, form)
            ev[2 * k + 1].record(s)
        torch.cuda.synchronize()
        ms = float(np.mean([ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(steps)]))
        res[form] = {"ms_per_launch": round(ms, 4), "tflops": round(alg / (ms * 1e-3) / 1e12, 4),
                     "us_per_theta": round(ms * 1e3 / len(sites), 4)}
    # tcgen05 kind::tf32 peak: one CTA per SM, 16384 M128 N256 K8 MMAs each
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sink = torch.zeros(sms, dtype=torch.float64, device=dev)
    iters = 16384
    for _ in range(2):
        _lib.check(lib.mpsb_tf32_probe(iters, sms, sink.data_ptr(), s.cuda_stream), "tf32 probe")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    _lib.check(lib.mpsb_tf32_probe(iters, sms, sink.data_ptr(), s.cuda_stream), "tf32 probe")
    e1.record(s)
    torch.cuda.synchronize()
    tf32_peak = 2.0 * 128 * 256 * 8 * iters * sms / (e0.elapsed_time(e1) * 1e-3) / 1e12
    mixed_s = res["mixed"]["ms_per_launch"] * 1e-3
    res["mixed"].update({"tensor_tflops_issued": round(issued / mixed_s / 1e12, 4),
                         "frac_of_tf32_peak": round(issued / mixed_s / 1e12 / tf32_peak, 5)})
    res["fp64"]["frac_of_fp64_peak"] = round(res["fp64"]["tflops"] / fp64_peak_tflops, 5)
    res["tf32_peak_tflops"] = round(tf32_peak, 3)
    res["tf32_peak_source"] = "measured: tcgen05 kind::tf32 probe (mpsb_tf32_probe), one CTA per SM, burst"
    res["share_of_an_update"] = {form: round(res[form]["us_per_theta"] * 1e-6 / update_s_per_update, 4)
                                 for form in ("fp64", "mixed")}
    res["note"] = ("tflops = algorithmic contraction+gate flops (32 chi_l chi_m chi_r + 128 chi_l chi_r per pair) "
                   "per second; tensor_tflops_issued counts the 9 real TF32 GEMMs (3M x 3xTF32) with padding; "
                   "share_of_an_update = theta time per pair / update time per pair in the per-layer launches "
                   "(the update kernel runs the same code as its phase 1, two CTAs per pair)")
    del tb
    return res


def cpu_baseline_sample(workers: int):
    from oracle.cpu_baseline import make_pool, run_parallel, single_process_default_threads
    pool = make_pool(workers)
    try:
        run_parallel(8, 2, 4, CUTOFF, workers, seed=SEED, pool=pool)  # spawn + import outside the timing
        r = run_parallel(N_SITES, DEPTH, CHI, CUTOFF, workers, reps=1, seed=SEED, pool=pool)
    finally:
        pool.close()
        pool.join()
    one = single_process_default_threads(CHI, 40, SEED)
    # untimed: the oracle's own final state of the benchmark circuit (seed SEED, as rank 0's),
    # the FP64 reference the device forms' infidelity is reported against
    ref = run_parallel(N_SITES, DEPTH, CHI, CUTOFF, 1, reps=1, seed=SEED, keep_first=True)
    return {"_final": (ref["final_sites"], ref["final_norm_log"]),
            "value": round(r["updates_per_s"], 3), "unit": UNIT, "cores": workers, "kind": "port",
            "sample": (f"{workers} single-BLAS-thread processes, each one full n={N_SITES} depth-{DEPTH} "
                       f"chi={CHI} circuit ({r['updates']} updates, {r['wall_s']:.1f} s wall); oracle "
                       "restatement of mps_core.py with scipy gesdd"),
            "single_process_default_threads": {
                "value": round(one["updates_per_s"], 3), "unit": UNIT,
                "sample": f"{one['updates']} saturated chi={CHI} updates in one process, default BLAS threads"}}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.cpu_baseline import make_pool, run_parallel, usable_cores
    workers = usable_cores()
    pool = make_pool(workers)
    try:
        for _ in range(args.warmup):
            run_parallel(N_SITES, DEPTH, CHI, CUTOFF, workers, seed=SEED, pool=pool)
        t0 = time.perf_counter()
        total = 0
        for _ in range(args.steps):
            total += run_parallel(N_SITES, DEPTH, CHI, CUTOFF, workers, seed=SEED, pool=pool)["updates"]
        dt = time.perf_counter() - t0
    finally:
        pool.close()
        pool.join()
    value = total / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Haar gates)",
            "config": {"workload": WORKLOAD, "parallelism": f"{workers} host processes x 1 circuit each"},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": workers, "kind": "port",
                             "sample": f"{workers} processes x one full circuit per step"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU side
def run_ours(args) -> None:
    import torch
    from fpga_mps_simulator_b200 import MPSBatch, MPSState, _lib
    from fpga_mps_simulator_b200.circuits import brickwall_layers

    from fpga_mps_simulator_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    reps = Replicas("nccl", dev, timeout_s=300)
    world, rank = reps.world, reps.rank
    lib = _lib.load()
    precision = args.precision

    # ---- CPU baseline first (spawned workers, before heavy GPU work; rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle.cpu_baseline import usable_cores
        cpu = cpu_baseline_sample(usable_cores())

    layers = brickwall_layers(N_SITES, DEPTH, reps.seed(SEED))
    n_upd = sum(len(L.sites) for L in layers)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def reset(b):
        b.sites.zero_()
        b.sites[:, 0] = 1.0
        b.bonds.fill_(1)
        b.norm_logs.zero_()
        b.status_acc.zero_()

    barrier = reps.barrier
    max_over_ranks = reps.max

    # ---- FP64 peak probe (the roofline denominator for the FP64-bound kernel)
    props = torch.cuda.get_device_properties(dev)
    sink = torch.zeros(1, dtype=torch.float64, device=dev)
    probe_blocks, probe_threads, probe_iters = props.multi_processor_count * 8, 256, 1 << 16
    s = torch.cuda.current_stream(dev)
    for _ in range(2):
        _lib.check(lib.mpsb_fp64_probe(probe_iters, probe_blocks, probe_threads, sink.data_ptr(), s.cuda_stream),
                   "fp64 probe")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    _lib.check(lib.mpsb_fp64_probe(probe_iters, probe_blocks, probe_threads, sink.data_ptr(), s.cuda_stream),
               "fp64 probe")
    e1.record()
    torch.cuda.synchronize()
    fp64_peak_tflops = probe_blocks * probe_threads * probe_iters * 16.0 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    gpu_id = "GPU-" + str(props.uuid) if hasattr(props, "uuid") else str(local)

    def measure(precision: str, timed: bool):
        """Warm-up, then K device-timed steps of one form; returns stats and the final state."""
        tol = args.mixed_tol if precision == "mixed" else 0.0
        batch = MPSBatch([N_SITES], [CHI], [CUTOFF], precision=precision, device=dev, tol=tol)
        pbs = [batch.make_pairs(np.zeros(len(L.sites), np.int32), L.sites, L.gates) for L in layers]
        for _ in range(args.warmup):
            reset(batch)
            for pb in pbs:
                batch.run_pairs(pb)
        torch.cuda.synchronize()
        batch.check_status()
        clocks = ClockSampler(gpu_id) if timed else None
        barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.begin()
        step_ms, layer_ms = [], np.zeros(len(layers))
        for _ in range(args.steps):
            flush.zero_()
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(layers) + 2)]
            evs[0].record()
            reset(batch)
            evs[1].record()
            for li, pb in enumerate(pbs):
                batch.run_pairs(pb)
                evs[li + 2].record()
            torch.cuda.synchronize()
            step_ms.append(evs[0].elapsed_time(evs[-1]))
            for li in range(len(layers)):
                layer_ms[li] += evs[li + 1].elapsed_time(evs[li + 2])
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop() if clocks else None
        batch.check_status()
        total_s = max_over_ranks(sum(step_ms) * 1e-3)
        kept = [pb.kept.cpu().numpy() for pb in pbs]
        dims = replay_dims(N_SITES, [L.sites for L in layers], kept)
        flops = sum(update_flops(cl, cm, cr) for per in dims for cl, cm, cr, _ in per)
        hbm = sum(update_bytes(cl, cm, cr, k) for per in dims for cl, cm, cr, k in per)
        kern_s = layer_ms.sum() * 1e-3 / args.steps
        trunc = np.concatenate([pb.trunc.cpu().numpy() for pb in pbs])  # discarded weight per update
        return {"batch": batch, "value": world * n_upd * args.steps / total_s, "total_s": total_s,
                "flops": flops, "hbm": hbm, "kern_s": kern_s, "clocks": clk,
                "achieved_tf": flops / kern_s / 1e12, "trunc": trunc,
                "layer_ms": [round(float(v) / args.steps, 4) for v in layer_ms]}

    # per-layer launches (one launch per layer), both forms: the reference point and the state checks
    main = measure(precision, timed=False)
    other_prec = "fp64" if precision == "mixed" else "mixed"
    other = measure(other_prec, timed=False)

    def measure_flow(prec: str, timed: bool, ref: dict):
        """The same circuit as ONE dataflow launch (all 20 layers; each pair starts when its two
        predecessors are done), device-timed like the per-layer steps: reset + launch per step,
        L2 flushed before each; the launch alone is timed for the roofline."""
        batch = MPSBatch([N_SITES], [CHI], [CUTOFF], precision=prec, device=dev,
                         tol=args.mixed_tol if prec == "mixed" else 0.0)
        fb = batch.make_flow(np.concatenate([np.zeros(len(L.sites), np.int32) for L in layers]),
                             np.concatenate([L.sites for L in layers]), np.concatenate([L.gates for L in layers]))
        for _ in range(args.warmup):
            reset(batch)
            batch.run_flow(fb)
        torch.cuda.synchronize()
        batch.check_status()
        clocks = ClockSampler(gpu_id) if timed else None
        barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.begin()
        step_ms, kern_ms = [], []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            reset(batch)
            e1.record()
            batch.run_flow(fb)
            e2.record()
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e2))
            kern_ms.append(e1.elapsed_time(e2))
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop() if clocks else None
        batch.check_status()
        total_s = max_over_ranks(sum(step_ms) * 1e-3)
        kern_s = sum(kern_ms) * 1e-3 / args.steps
        same = all(torch.equal(x, y) for x, y in zip(batch.snapshot(), ref["batch"].snapshot()))
        return {"value": world * n_upd * args.steps / total_s, "total_s": total_s, "kern_s": kern_s,
                "clocks": clk, "achieved_tf": ref["flops"] / kern_s / 1e12, "bitwise_equal_to_per_layer": same}

    fmain = measure_flow(precision, True, main)
    fother = measure_flow(other_prec, False, other)
    value, total_s = fmain["value"], fmain["total_s"]
    mixed_v, fp64_v = (value, fother["value"]) if precision == "mixed" else (fother["value"], value)
    flops, hbm, kern_s, achieved_tf, clk = main["flops"], main["hbm"], fmain["kern_s"], fmain["achieved_tf"], fmain["clocks"]
    flow = {"per_layer_launches": {precision: round(main["value"], 3), other_prec: round(other["value"], 3)},
            f"{precision}_ms_per_layer_launch": main["layer_ms"],
            "one_dataflow_launch": {precision: round(value, 3), other_prec: round(fother["value"], 3)},
            f"{precision}_bitwise_equal": fmain["bitwise_equal_to_per_layer"],
            f"{other_prec}_bitwise_equal": fother["bitwise_equal_to_per_layer"],
            "note": ("value = one dataflow launch per step (all 20 layers: a cluster per update, claimed in "
                     "layer order, started when its two predecessors finish, + one norm_log fold); "
                     "per_layer_launches = 20 launches per step, each layer's pairs in one; final states "
                     "compared bit for bit")}
    from fpga_mps_simulator_b200.mps import overlap
    ab, lab = overlap(main["batch"], 0, other["batch"], 0)
    aa, laa = overlap(main["batch"], 0, main["batch"], 0)
    bb, lbb = overlap(other["batch"], 0, other["batch"], 0)
    infid = 1.0 - abs(ab) ** 2 / (aa.real * bb.real) * math.exp(2 * lab - laa - lbb)
    batch = main["batch"]
    # per-update truncation error (discarded weight) of both forms, and <Z_i> on every site
    zop = np.diag([1.0, -1.0]).astype(np.complex128)
    zterms = [(i, zop, None) for i in range(N_SITES)]
    z_main = main["batch"].expect_terms(zterms)[0]
    z_other = other["batch"].expect_terms(zterms)[0]
    # both forms against the oracle's final state of the same circuit (the FP64 reference of
    # the metric), overlaps taken on the device
    vs_oracle = None
    if cpu is not None and cpu.get("_final") is not None:
        sites_ref, nl_ref = cpu.pop("_final")
        rb = MPSBatch([N_SITES], [CHI], [CUTOFF], precision="fp64", device=dev)
        for k, t in enumerate(sites_ref):
            rb.set_site(0, k, t)
        rb.norm_logs.fill_(nl_ref)
        rr, lrr = overlap(rb, 0, rb, 0)
        vs_oracle = {}
        for name, res in ((precision, main), (other_prec, other)):
            xb, lxb = overlap(res["batch"], 0, rb, 0)
            xx, lxx = overlap(res["batch"], 0, res["batch"], 0)
            vs_oracle[name] = 1.0 - abs(xb) ** 2 / (xx.real * rr.real) * math.exp(2 * lxb - lxx - lrr)
        vs_oracle["note"] = ("final state of each device form against the oracle's (mps_core semantics, "
                             "scipy gesdd, FP64) final state of the same circuit")
        del rb
    tr_m, tr_o = main["trunc"], other["trunc"]
    form_errors = {"discarded_weight_per_update": {f"{precision}_mean": float(tr_m.mean()),
                                                   f"{other_prec}_mean": float(tr_o.mean()),
                                                   "max_abs_diff": float(np.max(np.abs(tr_m - tr_o)))},
                   "z_expectation_max_abs_diff": float(np.max(np.abs(z_main - z_other)))}
    if vs_oracle is not None:
        form_errors["infidelity_vs_oracle"] = vs_oracle

    # ---- mixed vs FP64 state infidelity as the circuit deepens (untimed replay)
    by_depth = {}
    if not args.quick:
        forms = {}
        for prec in ("mixed", "fp64"):
            b2 = MPSBatch([N_SITES], [CHI], [CUTOFF], precision=prec, device=dev,
                          tol=args.mixed_tol if prec == "mixed" else 0.0)
            forms[prec] = (b2, [b2.make_pairs(np.zeros(len(L.sites), np.int32), L.sites, L.gates) for L in layers])
        for li in range(len(layers)):
            for prec, (b2, pbs2) in forms.items():
                b2.run_pairs(pbs2[li])
            if (li + 1) % 5 == 0:
                bm, bf = forms["mixed"][0], forms["fp64"][0]
                ab, lab = overlap(bm, 0, bf, 0)
                aa, laa = overlap(bm, 0, bm, 0)
                bb, lbb = overlap(bf, 0, bf, 0)
                by_depth[li + 1] = 1.0 - abs(ab) ** 2 / (aa.real * bb.real) * math.exp(2 * lab - laa - lbb)
        for b2, _ in forms.values():
            b2.check_status()
        forms.clear()

    # ---- the contraction alone (both forms) against its own rooflines
    contraction = None
    if not args.quick:
        contraction = contraction_leg(dev, main["batch"], np.concatenate([L.gates for L in layers]), 5,
                                      fp64_peak_tflops, main["kern_s"] / n_upd)

    # ---- the drop-in called gate by gate, as mps_core users write it (FP64): the whole
    # circuit as 990 MPSState._apply_adjacent_2q calls, then a read (flush), wall-clocked
    # from the first call to the synchronised result; deferred (default) and eager
    single = None
    if not args.quick:
        calls = [(int(i), g) for L in layers for i, g in zip(L.sites, L.gates)]
        runs = {}
        for defer in (True, False):
            for timed_run in (False, True):  # the first run sizes workspaces and kernel attributes
                st1 = MPSState(N_SITES, CHI, CUTOFF, precision="fp64", device=dev, defer=defer)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for i, g in calls:
                    st1._apply_adjacent_2q(i, g)
                st1.flush()
                torch.cuda.synchronize()
                wall = time.perf_counter() - t0
            st1.check_status()
            runs[defer] = (len(calls) / wall, st1)
        same = all(torch.equal(x, y) for x, y in zip(runs[True][1]._b.snapshot(), runs[False][1]._b.snapshot()))
        single = {"updates_per_s": round(runs[True][0], 3),
                  "eager_updates_per_s": round(runs[False][0], 3),
                  "bitwise_equal": bool(same),
                  "note": ("plain complex128 drop-in called gate by gate (990 MPSState._apply_adjacent_2q calls of "
                           "this circuit, then a read), wall clock: updates_per_s with the calls queued and run as one "
                           "dataflow launch at the read (the default), eager_updates_per_s with one launch per call")}
        del runs

    # ---- end to end through the public API, gates from pinned host memory, MPS read back
    e2e = None
    if not args.quick:
        st = MPSState(N_SITES, CHI, CUTOFF, precision=precision, device=dev)
        pinned = torch.from_numpy(np.ascontiguousarray(np.concatenate([L.gates for L in layers]))).pin_memory()
        ones = torch.ones(N_SITES, dtype=torch.complex128).pin_memory()
        out_sites = torch.empty(st._b.sites.shape, dtype=torch.complex128).pin_memory()
        out_bonds = torch.empty(N_SITES + 1, dtype=torch.int32).pin_memory()
        out_nl = torch.empty(1, dtype=torch.float64).pin_memory()
        h2d = pinned.numel() * 16 + N_SITES * 16
        d2h = out_sites.numel() * 16 + out_bonds.numel() * 4 + 8
        flow_tables = [None]  # built by the first (untimed) call, then reused: only the gates travel

        def e2e_step():
            b = st._b
            b.sites.zero_()
            b.sites[:, 0].copy_(ones, non_blocking=True)
            b.bonds.fill_(1)
            b.norm_logs.zero_()
            flow_tables[0] = st.apply_layers([L.sites for L in layers], pinned, flow=flow_tables[0])
            out_sites.copy_(b.sites, non_blocking=True)
            out_bonds.copy_(b.bonds, non_blocking=True)
            out_nl.copy_(b.norm_logs, non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        st.check_status()
        e2e = {"value": round(world * n_upd * args.steps / e2e_s, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    batching = None
    if not args.quick and not args.no_batching:
        batching = batching_leg(dev, 2, rank, max_over_ranks)
    large = large_leg(dev) if not (args.quick or args.no_large) else None
    gradient = None
    if not args.quick and not args.no_gradient:
        from oracle.cpu_baseline import usable_cores
        cw = usable_cores() if (rank == 0 and world == 1 and not args.no_cpu) else 0
        torch.cuda.empty_cache()  # the 7.6 GB of tapes below should not fight the earlier legs' cached blocks
        gradient = gradient_leg(dev, 5, 5, rank, max_over_ranks, cpu_workers=cw)
        for key in ("fp64", "mixed", "mixed_all", "fp64_checkpointed"):  # fraction of the same FP64 roofline
            gradient[key]["roofline_frac"] = round(gradient[key]["achieved_tflops"] / fp64_peak_tflops, 4)

    reps.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_s * 1e3 / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == "fp64" else "f64+tf32x3",
        "forms": {precision: round(value, 3), other_prec: round(fother["value"], 3),
                  "infidelity_mixed_vs_fp64": infid, **form_errors,
                  "infidelity_mixed_vs_fp64_by_depth": by_depth,
                  "launch_modes": flow,
                  "note": "batched per layer; mixed = 3xTF32 tcgen05 complex-3M theta + FP64 Jacobi SVD"},
        "target_ratio": {
            "batched_mixed_over_batched_fp64": round(mixed_v / fp64_v, 3),
            "batched_mixed_over_per_update_fp64": (round(mixed_v / single["eager_updates_per_s"], 2)
                                                   if single else None),
            "batched_mixed_over_deferred_drop_in_fp64": (round(mixed_v / single["updates_per_s"], 2)
                                                         if single else None),
            "target": ">= 5x the plain complex128 GPU form at infidelity <= 1e-6",
            "note": ("first reading: both forms batched, one dataflow launch each (the mixed form moves only the "
                     "contraction, 1-2 % of an update (the contraction leg), onto the tensor cores; the FP64 Jacobi SVD is the rest); "
                     "second reading: the plain form as the drop-in runs it one update per launch; third: the "
                     "drop-in called gate by gate with its calls queued into one dataflow launch")},
        "data": "synthetic (seeded Haar-random 4x4 gates, |0...0> start)",
        "config": {"workload": WORKLOAD, "precision": precision, "updates_per_step": n_upd,
                   "launches_per_step": 2, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "flushed between steps (256 MiB write)"},
        "roofline": {"bound": "fp64", "achieved": round(achieved_tf, 4), "peak": round(fp64_peak_tflops, 4),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / fp64_peak_tflops, 4),
                     "traffic": TRAFFIC_PER_LAUNCH, "traffic_source": TRAFFIC_SOURCE,
                     "peak_source": "measured: FP64 FMA probe (mpsb_fp64_probe) on this GPU, burst",
                     "kernel": f"update2q_flow_kernel ({precision}) + fold_flow_kernel",
                     "flops_per_step": flops, "hbm_site_bytes_per_step": hbm,
                     "hbm_gbs": round(hbm / kern_s / 1e9, 3)},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
        "e2e": e2e,
        "per_update_path": single,
        "contraction": contraction,
        "batching": batching,
        "gradient": gradient,
        "large": large,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_leg(args) -> None:
    """One secondary leg alone on GPU 0 (for profiling); prints its JSON object."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ident = lambda x: x  # noqa: E731  (one rank: the max over ranks is the value itself)
    if args.leg == "gradient":
        res = gradient_leg(dev, args.steps, args.warmup, 0, ident)
    elif args.leg == "batching":
        res = batching_leg(dev, args.steps, 0, ident)
    elif args.leg == "contraction":
        from fpga_mps_simulator_b200 import MPSBatch
        from fpga_mps_simulator_b200.circuits import brickwall_layers
        layers = brickwall_layers(N_SITES, DEPTH, SEED)
        batch = MPSBatch([N_SITES], [CHI], [CUTOFF], precision="mixed", device=dev)
        for L in layers:
            batch.apply_layer(np.zeros(len(L.sites), np.int32), L.sites, L.gates)
        torch.cuda.synchronize()
        batch.check_status()
        res = contraction_leg(dev, batch, np.concatenate([L.gates for L in layers]), args.steps, float("nan"),
                              float("nan"))
    else:
        res = large_leg(dev)
    print(json.dumps({"leg": args.leg, **res}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed",
                    help="form of the headline value (the other form is reported beside it)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--quick", action="store_true", help="skip the e2e, per-update and batching legs")
    ap.add_argument("--mixed-tol", type=float, default=0.0,
                    help="Jacobi off-diagonal tolerance of the mixed form (0 = library default 1e-9)")
    ap.add_argument("--no-batching", action="store_true", help="skip the 256-circuit batching leg")
    ap.add_argument("--no-gradient", action="store_true", help="skip the ansatz energy-gradient leg")
    ap.add_argument("--leg", choices=["all", "gradient", "batching", "large", "contraction"], default="all",
                    help="run one secondary leg alone and print its JSON (profiling)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 1000-qubit XXZ initial-state gradient leg (about a minute)")
    ap.add_argument("--grad-vectors", type=int, default=64,
                    help="parameter vectors of the gradient leg (fewer: a small case for profiling)")
    args = ap.parse_args()
    globals()["GRAD_VEC"] = args.grad_vectors
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.leg != "all":
        run_leg(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
