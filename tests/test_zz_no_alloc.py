"""The allocation-free update entry point against the workspace entry point.

mpsb_update2q_batch_noalloc serves callers that cannot allocate device memory
(a host that only hands the library pre-registered buffers, or a loop where a
cudaMalloc would synchronise the device): it keeps its scratch in a fixed
16 MiB device array instead of a caller workspace.  This test drives both
entry points through the C ABI on identical chains, two calls in a row, and
requires the same spectra, kept counts, bonds, norm_log and amplitudes within
the FP64 parity tolerance, in both forms (at chi_cap = 64 the mixed form is the
tensor-core kernel with its own shared-memory size and cutoff floor); it also
checks that an oversized batch is refused
before anything is launched.  It lives in the last test file so that a run
stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_workspace_entry_two_calls(precision):
    from fpga_mps_simulator_b200 import MPSBatch, _lib
    from fpga_mps_simulator_b200.circuits import brickwall_layers

    lib = _lib.load()
    n, chi, cut = 24, 64, 1e-10
    code = _lib.FP64 if precision == "fp64" else _lib.MIXED_TF32X3
    ref = MPSBatch([n], [chi], [cut], precision=precision)
    new = MPSBatch([n], [chi], [cut], precision=precision)
    layers = brickwall_layers(n, 8, 321)
    # bring both chains to a saturated state the same way
    for L in layers[:6]:
        ref.apply_layer(np.zeros(len(L.sites), np.int32), L.sites, L.gates)
        new.apply_layer(np.zeros(len(L.sites), np.int32), L.sites, L.gates)
    stream = torch.cuda.current_stream().cuda_stream
    for L in layers[6:8]:  # two calls in a row through each entry point
        pa = ref.make_pairs(np.zeros(len(L.sites), np.int32), L.sites, L.gates, record_spectra=True)
        ref.run_pairs(pa)
        pb = new.make_pairs(np.zeros(len(L.sites), np.int32), L.sites, L.gates, record_spectra=True)
        rc = lib.mpsb_update2q_batch_noalloc(new.table.data_ptr(), pb.pairs.data_ptr(), pb.npairs,
                                             pb.gates.data_ptr(), code, new.chi_cap, 0.0, 0,
                                             pb.spectra.data_ptr(), pb.kept.data_ptr(), pb.trunc.data_ptr(),
                                             pb.status.data_ptr(), stream)
        _lib.check(rc, "mpsb_update2q_batch_noalloc")
        torch.cuda.synchronize()
        sa, sb = pa.spectra.cpu().numpy(), pb.spectra.cpu().numpy()
        np.testing.assert_allclose(sb, sa, rtol=0, atol=TOL * sa.max())
        assert np.array_equal(pa.kept.cpu().numpy(), pb.kept.cpu().numpy())
        assert not pb.status.any().item()
        np.testing.assert_allclose(pb.trunc.cpu().numpy(), pa.trunc.cpu().numpy(), rtol=0, atol=TOL)
    ref.check_status()
    new.check_status()
    assert new.bond_dims(0) == ref.bond_dims(0)
    assert abs(new.norm_log(0) - ref.norm_log(0)) < TOL * max(1.0, abs(ref.norm_log(0)))
    bits = np.random.default_rng(0).integers(0, 2, size=(16, n))
    a_ref, a_new = ref.amplitudes(0, bits), new.amplitudes(0, bits)
    np.testing.assert_allclose(a_new, a_ref, rtol=0, atol=TOL * np.abs(a_ref).max())


def test_noalloc_rejects_batches_beyond_its_scratch():
    from fpga_mps_simulator_b200 import _lib
    lib = _lib.load()
    too_many = 64  # 64 pairs at chi_cap 64 need 16 MiB of theta copies plus the records
    assert lib.mpsb_update2q_workspace_bytes(too_many, 64) > (16 << 20)
    rc = lib.mpsb_update2q_batch_noalloc(256, 256, too_many, 256, _lib.FP64, 64, 0.0, 0,
                                         None, None, None, 256, None)
    assert rc == -3
    assert b"scratch" in lib.mpsb_last_error()
