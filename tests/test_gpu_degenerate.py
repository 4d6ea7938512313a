"""Parity of the two-site update on theta with degenerate and tightly
clustered singular values, where one-sided Jacobi converges slowest and where
the sweeps' stopping rule (stop after a sweep whose rotations were all below
sqrt(2 tol) in relative |x^H y|) has the least margin.

theta is built with a prescribed spectrum: M = U diag(s) V^H, split as
A = U sqrt(s), B = sqrt(s) V^H over a bond of dimension rank(M), gate = I, so
the update factorises exactly M (mps_core.py:326-350 semantics, oracle
update_forward).  Checked on the gauge-invariant A'B', the kept count and the
spectrum against the oracle.  Truncations fall only in gaps of the spectrum,
so the kept subspace is well defined.
"""
import numpy as np
import pytest
import torch

from oracle.mps_adjoint import update_forward

pytestmark = pytest.mark.gpu


def _haar(rng, n):
    q, r = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return q * (np.diag(r) / np.abs(np.diag(r)))[None, :]


def _sites(rng, cl, cr, s):
    """A (cl, 2, k), B (k, 2, cr) with A B = U diag(s) V^H as a (2cl) x (2cr) matrix."""
    k = len(s)
    U = _haar(rng, 2 * cl)[:, :k]
    V = _haar(rng, 2 * cr)[:, :k]
    A = (U * np.sqrt(s)[None, :]).reshape(cl, 2, k)
    B = (np.sqrt(s)[:, None] * V.conj().T).reshape(k, 2, cr)
    return A, B


SPECTRA = {
    # name: (chi_l, chi_r, spectrum, chi_max, relative cutoff)
    # exact degeneracies, all kept
    "blocks_16": (8, 8, np.repeat([1.0, 0.5, 0.25, 1e-3], 4), 16, 1e-12),
    "blocks_32": (16, 16, np.repeat([1.0, 0.5, 0.25, 1e-3], 8), 32, 1e-12),
    # clusters 1e-9 apart, truncated by the cutoff in the gap between the clusters
    "clusters_cut": (16, 16, np.concatenate([1.0 + 1e-9 * np.arange(12), 0.3 + 1e-9 * np.arange(4),
                                             1e-2 + 1e-10 * np.arange(16)]), 32, 0.05),
    # rank-deficient 128 x 128 theta: 64 nonzero values in four degenerate
    # groups and 64 exact zeros, all nonzero ones kept
    "blocks_64_rank_deficient": (64, 64, np.repeat([1.0, 0.7, 0.2, 0.05], 16), 64, 1e-12),
    # a flat spectrum with one gap, truncated there by the cutoff
    "flat_cut_64": (64, 64, np.concatenate([1.0 + 1e-8 * np.arange(40), 0.1 * (1.0 + 1e-8 * np.arange(24))]), 64, 0.5),
}


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(SPECTRA))
def test_degenerate_spectrum_update_matches_oracle(name, prec):
    from fpga_mps_simulator_b200 import MPSBatch
    cl, cr, s, chi_max, cut = SPECTRA[name]
    rng = np.random.default_rng(sorted(SPECTRA).index(name) + 77)
    A, B = _sites(rng, cl, cr, np.asarray(s, float))
    G = np.eye(4, dtype=np.complex128)
    b = MPSBatch([16], [chi_max], [cut], precision=prec)
    b.set_site(0, 7, A)
    b.set_site(0, 8, B)
    pb = b.apply_layer([0], [7], G[None], record_spectra=True)
    torch.cuda.synchronize()
    b.check_status()
    rA, rB, aux = update_forward(A, B, G, chi_max, cut)
    got = np.einsum("lpm,mqr->lpqr", b.site(0, 7), b.site(0, 8))
    want = np.einsum("lpm,mqr->lpqr", rA, rB)
    scale = max(1.0, float(np.max(np.abs(want))))
    if prec == "fp64":
        assert int(pb.kept.item()) == aux["keep"]
        assert float(np.max(np.abs(got - want))) <= 1e-10 * scale
        S_ref = np.asarray(aux["S"])
        S_got = pb.spectra.cpu().numpy()[0][: len(S_ref)]
        assert float(np.max(np.abs(S_got - S_ref))) <= 1e-10 * S_ref[0]
    else:  # 3xTF32 theta at chi_cap 64 (the exact FP64 contraction below): state to ~1e-6
        assert float(np.max(np.abs(got - want))) <= 1e-5 * scale
