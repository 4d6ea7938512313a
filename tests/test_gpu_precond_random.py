"""Randomised parity of the QR-preconditioned update (graded theta: columns
sorted, blocked Householder QR over the cluster, Jacobi on R^H) against the
oracle's update (mps_core.py:326-350 semantics): 40 seeded shapes with bonds
up to 64 -- tall and wide theta, odd sizes that leave a QR panel partly
padding, unitary and non-unitary gates, both precisions -- checked on the
gauge-invariant product A'B' and the kept count."""
import numpy as np
import pytest
import torch

from oracle.mps_adjoint import update_forward

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(2026)
    out = []
    while len(out) < 40:
        cl, cm, cr = (int(x) for x in rng.integers(9, 65, size=3))
        chi = 64 if max(cl, cm, cr) > 32 else 32
        decay = float(rng.uniform(1.0, 3.0))  # decades the site scalings span
        prec = "mixed" if len(out) % 4 == 3 else "fp64"
        out.append((len(out), cl, cm, cr, chi, decay, bool(len(out) % 3 == 1), prec))
    return out


@pytest.mark.parametrize("seed,cl,cm,cr,chi,decay,general,prec", _cases())
def test_graded_update_matches_oracle(seed, cl, cm, cr, chi, decay, general, prec):
    from fpga_mps_simulator_b200 import MPSBatch
    rng = np.random.default_rng(1000 + seed)
    A = rng.standard_normal((cl, 2, cm)) + 1j * rng.standard_normal((cl, 2, cm))
    B = rng.standard_normal((cm, 2, cr)) + 1j * rng.standard_normal((cm, 2, cr))
    A *= np.logspace(0.0, -decay, cl)[:, None, None]
    B *= np.logspace(0.0, -decay, cr)[None, None, :]
    G, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
    if general:
        G = G + 0.3 * (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
    cut = 1e-12
    b = MPSBatch([16], [chi], [cut], precision=prec)
    b.set_site(0, 7, A)
    b.set_site(0, 8, B)
    pb = b.apply_layer([0], [7], G[None])
    torch.cuda.synchronize()
    b.check_status()
    rA, rB, aux = update_forward(A, B, G, chi, cut)
    got = np.einsum("lpm,mqr->lpqr", b.site(0, 7), b.site(0, 8))
    want = np.einsum("lpm,mqr->lpqr", rA, rB)
    scale = max(1.0, float(np.max(np.abs(want))))
    if prec == "fp64":
        assert int(pb.kept.item()) == aux["keep"]
        assert float(np.max(np.abs(got - want))) <= 1e-10 * scale
    else:  # 3xTF32 theta at chi_cap 64 keeps nothing below 1e-6 S0; the state agrees to ~1e-6
        assert float(np.max(np.abs(got - want))) <= 1e-5 * scale
