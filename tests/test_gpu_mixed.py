"""GPU tests of the mixed-precision form (3xTF32 complex-3M tensor-core theta,
FP64 Jacobi SVD).  Tolerances: per-update singular values within 1e-5 * S[0]
of the FP64 reference, and state infidelity <= 1e-6 against the FP64 result
-- the error budget of the mixed form.  On the 100-site chi=64 circuit the
measured infidelity is ~9e-7: the error is dominated by how strongly the
chi_max truncation (no spectral gap at chi = 64) reacts to theta's ~1e-7
relative rounding, accumulated over 990 updates."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle.mps_oracle import OracleMPS, infidelity
from fpga_mps_simulator_b200.circuits import brickwall_layers

pytestmark = pytest.mark.gpu
SV_TOL = 1e-5
INFID = 1e-6


def _sites(st):
    return [st.sites[k] for k in range(st.n)]


@pytest.mark.parametrize("precision", ["mixed", "mixed_all"])
@pytest.mark.parametrize("name", ["brick_n16_d10_chi16", "brick_n40_d16_chi32", "brick_n20_d12_chi64"])
def test_mixed_spectra_and_fidelity_on_golden(name, precision):
    """"mixed_all" runs the tensor cores at chi_cap 16 and 32 too (64-row MMA tiles)."""
    from fpga_mps_simulator_b200 import MPSState
    g = load_golden(name)
    n = int(g["n"])
    st = MPSState(n, int(g["chi_max"]), float(g["cutoff"]), precision=precision)
    ref = OracleMPS(n, int(g["chi_max"]), float(g["cutoff"]))
    k0 = 0
    layer_sites, layer_gates = [], []
    cur, used = [], set()
    for i, gm in zip(g["sites"], g["gates"]):
        i = int(i)
        if i in used or i - 1 in used or i + 1 in used:
            layer_sites.append([c[0] for c in cur]); layer_gates.append(np.stack([c[1] for c in cur]))
            cur, used = [], set()
        cur.append((i, gm)); used.add(i)
    layer_sites.append([c[0] for c in cur]); layer_gates.append(np.stack([c[1] for c in cur]))
    for sites, gates in zip(layer_sites, layer_gates):
        pb = st.apply_layer(sites, gates, record_spectra=True)
        for i, gm in zip(sites, gates):
            ref.apply_adjacent_2q(i, gm)
        spec = pb.spectra.cpu().numpy()
        for k in range(len(sites)):
            L = int(g["spec_len"][k0 + k])
            S = g["spectra"][k0 + k, :L]
            np.testing.assert_allclose(spec[k, :L], S, rtol=0, atol=SV_TOL * S[0])
        k0 += len(sites)
    st.check_status()
    assert infidelity(_sites(st), ref.sites) <= INFID


@pytest.mark.parametrize("chi", [8, 16, 32])
def test_mixed_all_runs_the_tensor_cores_below_chi_64(chi):
    """At chi_cap <= 32 "mixed" keeps the exact FP64 contraction (spectra equal to
    FP64 up to the Jacobi tolerance) while "mixed_all" takes the 64-row
    tensor-core tile: its theta rounding (~1e-7 relative) shows in the spectra,
    within the mixed form's 1e-5 S[0] budget."""
    from fpga_mps_simulator_b200 import MPSState
    n, depth = 12, 6
    layers = brickwall_layers(n, depth, 77 + chi)
    out = {}
    for prec in ("fp64", "mixed_all"):
        st = MPSState(n, chi, 1e-12, precision=prec)
        spec = [st.apply_layer(L.sites, L.gates, record_spectra=True).spectra.cpu().numpy() for L in layers]
        st.check_status()
        out[prec] = (np.concatenate(spec), st)
    a, b = out["fp64"][0], out["mixed_all"][0]
    s0 = np.max(a, axis=1, keepdims=True)
    diff = np.max(np.abs(a - b) / s0)
    assert 1e-12 < diff < SV_TOL, diff
    ref = OracleMPS(n, chi, 1e-12)
    for L in layers:
        for i, g in zip(L.sites, L.gates):
            ref.apply_adjacent_2q(int(i), g)
    assert infidelity(_sites(out["mixed_all"][1]), ref.sites) <= INFID


def test_mixed_precision_config_against_fp64():
    """n=100, depth 20, chi_max=64, cutoff 1e-10: mixed vs the FP64 GPU form (== oracle to 1e-10)."""
    from fpga_mps_simulator_b200 import MPSState
    n, depth, chi, cut = 100, 20, 64, 1e-10
    a = MPSState(n, chi, cut, precision="fp64")
    b = MPSState(n, chi, cut, precision="mixed")
    for L in brickwall_layers(n, depth, 2024):
        a.apply_layer(L.sites, L.gates)
        b.apply_layer(L.sites, L.gates)
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    assert a.bond_dims() == b.bond_dims()
    inf = infidelity(_sites(a), _sites(b))
    assert inf <= INFID, inf
    za, zb = a.expect_z_all(), b.expect_z_all()
    assert np.max(np.abs(za - zb)) < 1e-4  # local observables follow the state error (~sqrt(infidelity))


def test_mixed_shapes_and_noise_floor():
    """Small and odd chi caps, wide/tall thetas; an exactly rank-deficient
    circuit keeps its exact bond dimensions despite tf32 rounding."""
    from fpga_mps_simulator_b200 import MPSState, GATE_MATRICES, gate_1q
    for n, chi in [(2, 64), (3, 3), (9, 7), (12, 33)]:
        st = MPSState(n, chi, 1e-12, precision="mixed")
        ref = OracleMPS(n, chi, 1e-12)
        for L in brickwall_layers(n, 7, n * 31 + chi):
            st.apply_layer(L.sites, L.gates)
            for i, gm in zip(L.sites, L.gates):
                ref.apply_adjacent_2q(int(i), gm)
        st.check_status()
        sv, svr = st.get_statevector(), ref.statevector()
        f = abs(np.vdot(sv, svr)) ** 2 / (np.vdot(sv, sv).real * np.vdot(svr, svr).real)
        assert 1 - f <= INFID
    # GHZ chain: every bond is exactly 2
    n = 12
    st = MPSState(n, 16, 1e-12, precision="mixed")
    st.apply_1q(0, GATE_MATRICES["h"])
    for i in range(n - 1):
        st.apply_2q(i, i + 1, GATE_MATRICES["cx"])
    assert st.bond_dims() == [2] * (n - 1)
    sv = st.get_statevector()
    assert abs(abs(sv[0]) ** 2 - 0.5) < 1e-6 and abs(abs(sv[-1]) ** 2 - 0.5) < 1e-6
