"""Host logic of the multi-chain layer schedules (no GPU): every strategy
covers each chain's pairs of each layer exactly once, keeps a chain's pairs
contiguous and disjoint, and orders / groups chains as the strategy says."""
import numpy as np
import pytest

from fpga_mps_simulator_b200._lib import keep_limit
from fpga_mps_simulator_b200.circuits import random_circuit_batch
from fpga_mps_simulator_b200.mps import validate_pairs
from fpga_mps_simulator_b200.schedule import STRATEGIES, Schedule


class _FakePairs:
    def __init__(self, ns, ci, si, gates):
        validate_pairs(ns, np.asarray(ci), np.asarray(si))
        self.ci, self.si, self.gates = list(ci), list(si), np.asarray(gates)
        self.npairs = len(self.si)


class _FakeBatch:
    precision = "mixed"

    def __init__(self, specs):
        self.ns = [s.n for s in specs]
        self.chi_maxs = [s.chi_max for s in specs]
        self.caps = [keep_limit(s.n, s.chi_max) for s in specs]

    @property
    def nchains(self):
        return len(self.ns)

    def make_pairs(self, ci, si, gates, record_spectra=False):
        return _FakePairs(self.ns, ci, si, gates)


@pytest.fixture(scope="module")
def specs():
    return random_circuit_batch(24, seed=5, n_range=(6, 40), depth_range=(2, 9), chis=(4, 16, 64))


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_strategy_covers_every_pair_once(specs, strategy):
    b = _FakeBatch(specs)
    sch = Schedule(b, [s.layers for s in specs])
    plan = sch.launches(strategy)
    assert len(plan) == max(s.depth for s in specs)
    total = 0
    for L, launches in enumerate(plan):
        seen = {}
        for lc in launches:
            assert lc.chi_cap >= max(b.caps[c] for c in lc.pb.ci)
            for c, i, g in zip(lc.pb.ci, lc.pb.si, lc.pb.gates):
                assert (c, i) not in seen
                seen[(c, i)] = g
            total += lc.pb.npairs
        for c, s in enumerate(specs):
            if L < s.depth:
                for i, g in zip(s.layers[L].sites, s.layers[L].gates):
                    np.testing.assert_array_equal(seen.pop((c, int(i))), g)
        assert not seen
    assert total == sch.updates()


def test_lpt_orders_by_decreasing_cost_and_split_groups_by_cap(specs):
    b = _FakeBatch(specs)
    sch = Schedule(b, [s.layers for s in specs])
    for launches in sch.launches("lpt"):
        assert len(launches) == 1
        caps = [b.caps[c] for c in launches[0].pb.ci]
        assert caps == sorted(caps, reverse=True)
    for launches in sch.launches("split"):
        caps = [lc.chi_cap for lc in launches]
        assert caps == sorted(set(caps), reverse=True)
        for lc in launches:
            assert {b.caps[c] for c in lc.pb.ci} == {lc.chi_cap}


def test_unknown_strategy_rejected(specs):
    sch = Schedule(_FakeBatch(specs), [s.layers for s in specs])
    with pytest.raises(ValueError):
        sch.launches("greedy")


def test_signature_depends_on_chi_mix(specs):
    a = Schedule(_FakeBatch(specs), [s.layers for s in specs]).signature()
    b = Schedule(_FakeBatch(specs[:-3]), [s.layers for s in specs[:-3]]).signature()
    assert a != b
