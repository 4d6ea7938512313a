"""GPU tests of MPSSimulator.run (the counterpart of FPGAMPSSimulator.run):
12 seeded random circuits -- routing, reversed pairs, Toffolis, resets,
measured subsets -- run together as one batch; statevectors (up to the
global phase a reset fall-back leaves gauge dependent) and seeded counts
equal what the reference engine produced from the reference compiler's gate
list (tests/golden/compiler.npz)."""
import numpy as np
import pytest

from test_compiler_host import golden_circuits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fuse", [True, False])
def test_simulator_matches_reference_engine(fuse):
    from fpga_mps_simulator_b200.compiler import MPSSimulator
    circs = golden_circuits()
    g = circs[0][1]
    sim = MPSSimulator(chi_max=64, svd_cutoff=1e-12, fuse_1q=fuse)
    res = sim.run([c for c, _, _ in circs], shots=int(g["shots"]), seed=int(g["seed"]))
    assert res.success()
    for idx, (c, g, p) in enumerate(circs):
        sv = res.get_statevector(idx)
        want = g[p + "sv"]
        # a reset that falls back to |0> (site entirely in |1>) drops the site's
        # phase, which is SVD-gauge dependent: equal up to a global phase
        ov = np.vdot(sv, want)
        ph = ov / abs(ov) if abs(ov) > 0 else 1.0
        np.testing.assert_allclose(sv * ph, want, atol=1e-10 * max(1.0, np.max(np.abs(want))))
        counts = res.get_counts(idx)
        assert sorted(counts) == list(g[p + "count_keys"])
        assert [counts[k] for k in sorted(counts)] == list(g[p + "count_vals"])
        assert res.get_max_bond(idx) == max(res.get_bond_dims(idx) or [1])
    times = res.get_phase_times(0)
    assert times["launches"] > 0 and times["layers"] > 0


def test_single_circuit_and_no_measure_measures_all():
    from fpga_mps_simulator_b200.compiler import Circuit, MPSSimulator
    c = Circuit(3)
    c.h(0)
    c.cx(0, 1)
    c.cx(1, 2)
    res = MPSSimulator().run(c, shots=1024, seed=0)
    counts = res.get_counts()
    assert set(counts) <= {"000", "111"} and sum(counts.values()) == 1024
    assert counts.get("000", 0) + counts.get("111", 0) > 0.95 * 1024
