"""GPU tests of the overlap read-out (mpsb_overlap): <a|b> of two chains,
norm_log factors included, against the oracle's transfer-matrix overlap, for
uneven bond caps; the infidelity helper built on it."""
import math

import numpy as np
import pytest

from oracle.mps_oracle import OracleMPS, mps_overlap
from fpga_mps_simulator_b200.circuits import brickwall_layers

pytestmark = pytest.mark.gpu


def _pair(n, depth, chi, cut, seed):
    from fpga_mps_simulator_b200 import MPSState
    st = MPSState(n, chi, cut)
    ref = OracleMPS(n, chi, cut)
    for L in brickwall_layers(n, depth, seed):
        st.apply_layer(L.sites, L.gates)
        for i, g in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), g)
    return st, ref


@pytest.mark.parametrize("chi_a,chi_b", [(64, 64), (16, 64), (8, 4)])
def test_overlap_matches_oracle(chi_a, chi_b):
    from fpga_mps_simulator_b200.mps import overlap
    n = 30
    a, ra = _pair(n, 12, chi_a, 1e-10, 1)
    b, rb = _pair(n, 12, chi_b, 1e-10, 1)   # same circuit, different truncation
    got, glog = overlap(a._b, 0, b._b, 0)
    want, wlog = mps_overlap(ra.sites, rb.sites, ra.norm_log, rb.norm_log)
    g = got * math.exp(glog)
    w = want * math.exp(wlog)
    assert abs(g - w) <= 1e-10 * max(1.0, abs(w))
    # self overlap = squared norm
    s, slog = overlap(a._b, 0, a._b, 0)
    ws, wslog = mps_overlap(ra.sites, ra.sites, ra.norm_log, ra.norm_log)
    assert abs(s * math.exp(slog) - ws * math.exp(wslog)) <= 1e-10 * abs(ws * math.exp(wslog))


def test_infidelity_of_independent_circuits():
    from fpga_mps_simulator_b200.mps import infidelity
    from oracle.mps_oracle import infidelity as oracle_infidelity
    a, ra = _pair(12, 6, 64, 1e-12, 3)
    b, rb = _pair(12, 6, 64, 1e-12, 4)
    assert abs(infidelity(a, b) - oracle_infidelity(ra.sites, rb.sites)) < 1e-10
    assert abs(infidelity(a, a)) < 1e-12
