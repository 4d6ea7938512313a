"""GPU tests of multi-chain schedules: every launch strategy (one launch,
cost-ordered launch, one launch per bond-cap class on concurrent streams)
reproduces the oracle chain by chain, a captured CUDA graph replays the eager
result bit for bit, and the autotuner leaves the state untouched."""
import numpy as np
import pytest
import torch

from oracle.mps_oracle import OracleMPS, infidelity
from fpga_mps_simulator_b200.circuits import random_circuit_batch

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _specs():
    return random_circuit_batch(10, seed=11, n_range=(5, 13), depth_range=(3, 10), chis=(4, 8, 16))


def _oracles(specs, cutoff):
    out = []
    for s in specs:
        ref = OracleMPS(s.n, s.chi_max, cutoff)
        for L in s.layers:
            for i, g in zip(L.sites, L.gates):
                ref.apply_adjacent_2q(int(i), g)
        out.append(ref)
    return out


def _batch(specs, precision, cutoff):
    from fpga_mps_simulator_b200 import MPSBatch
    return MPSBatch([s.n for s in specs], [s.chi_max for s in specs], cutoff, precision=precision)


@pytest.mark.parametrize("strategy", ["single", "lpt", "split", "flow"])
def test_strategies_match_oracle(strategy):
    from fpga_mps_simulator_b200.schedule import Runner, Schedule
    specs = _specs()
    b = _batch(specs, "fp64", 1e-12)
    Runner(Schedule(b, [s.layers for s in specs]), strategy).run()
    torch.cuda.synchronize()
    b.check_status()
    for c, ref in enumerate(_oracles(specs, 1e-12)):
        assert b.bond_dims(c) == ref.bond_dims()
        assert abs(b.norm_log(c) - ref.norm_log) < TOL
        sv = ref.statevector()
        np.testing.assert_allclose(b.statevector(c), sv, rtol=0, atol=TOL * np.max(np.abs(sv)))


@pytest.mark.parametrize("strategy", ["lpt", "split", "flow"])
def test_graph_replay_is_bitwise_eager(strategy):
    from fpga_mps_simulator_b200.schedule import Runner, Schedule
    specs = _specs()
    b = _batch(specs, "mixed", 1e-10)
    sch = Schedule(b, [s.layers for s in specs])
    init = b.snapshot()
    r = Runner(sch, strategy)
    r.run()
    torch.cuda.synchronize()
    eager = b.snapshot()
    b.restore(init)
    r.capture()
    for _ in range(2):  # a graph replays from whatever state it finds
        b.restore(init)
        r.run()
        torch.cuda.synchronize()
        b.check_status()
        for x, y in zip(b.snapshot(), eager):
            assert torch.equal(x, y)
    r.release()


def test_mixed_batch_fidelity_against_oracle():
    from fpga_mps_simulator_b200.schedule import Runner, Schedule
    specs = _specs()
    b = _batch(specs, "mixed", 1e-10)
    Runner(Schedule(b, [s.layers for s in specs]), "split").run()
    torch.cuda.synchronize()
    b.check_status()
    for c, ref in enumerate(_oracles(specs, 1e-10)):
        sites = [b.site(c, k) for k in range(specs[c].n)]
        assert infidelity(sites, ref.sites) <= 1e-6


def test_autotune_restores_state_and_caches():
    from fpga_mps_simulator_b200.schedule import STRATEGIES, Schedule, autotune, _TUNE_CACHE
    specs = _specs()
    b = _batch(specs, "mixed", 1e-10)
    sch = Schedule(b, [s.layers for s in specs])
    before = b.snapshot()
    best = autotune(sch, start=2, layers=3, repeats=1)
    torch.cuda.synchronize()
    assert best in STRATEGIES
    for x, y in zip(before, b.snapshot()):
        assert torch.equal(x, y)
    assert autotune(sch, start=2, layers=3, repeats=1) == best
    assert (sch.signature(), 2, 3) in _TUNE_CACHE
