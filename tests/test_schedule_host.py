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


def test_flow_items_dependencies_are_the_last_earlier_touch():
    from fpga_mps_simulator_b200.mps import flow_items
    # chain 0 (n=6): (0,1) (2,3) (4,5) | (1,2) (3,4) ; chain 1 (n=4): (0,1) (2,3) | (1,2)
    ci = [0, 0, 0, 1, 1, 0, 0, 1]
    si = [0, 2, 4, 0, 2, 1, 3, 1]
    items, order, off = flow_items([6, 4], ci, si)
    assert items[:, 2].tolist() == list(range(8)) and items[:, 3].tolist() == list(range(8))
    deps = {k: (int(items[k, 4]), int(items[k, 5])) for k in range(8)}
    assert deps[0] == deps[1] == deps[2] == deps[3] == deps[4] == (-1, -1)
    assert deps[5] == (0, 1) and deps[6] == (1, 2) and deps[7] == (3, 4)
    assert all(d < k for k, ds in deps.items() for d in ds)  # topological
    assert off.tolist() == [0, 5, 8]
    assert order[:5].tolist() == [0, 1, 2, 5, 6] and order[5:].tolist() == [3, 4, 7]
    with pytest.raises(ValueError, match="range"):
        flow_items([6], [0], [5])


def test_flow_plan_lists_each_class_layer_by_layer(specs):
    class _Fake(_FakeBatch):
        def make_flow(self, ci, si, gates, record_spectra=False):
            from fpga_mps_simulator_b200.mps import flow_items
            flow_items(self.ns, ci, si)
            return _FakePairs.__new__(_FakePairs), (list(ci), list(si), np.asarray(gates))

    b = _Fake(specs)
    sch = Schedule(b, [s.layers for s in specs])
    plan = sch.flow_plan()
    assert [fl.chi_cap for fl in plan] == sorted(set(b.caps), reverse=True)
    total = 0
    for fl in plan:
        ci, si, gates = fl.fb[1]
        total += len(ci)
        assert {b.caps[c] for c in ci} == {fl.chi_cap}
        for c in set(ci):  # a chain's updates in layer order, each layer in its own order
            mine = [(s, g) for cc, s, g in zip(ci, si, gates) if cc == c]
            want = [(int(i), g) for L in specs[c].layers for i, g in zip(L.sites, L.gates)]
            assert [s for s, _ in mine] == [s for s, _ in want]
            for (_, g1), (_, g2) in zip(mine, want):
                np.testing.assert_array_equal(g1, g2)
    assert total == sch.updates()


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
