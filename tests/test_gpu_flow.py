"""The dataflow launch (mpsb_update2q_flow): many layers of many chains in one
launch, each update starting once the two updates it depends on are done.

* It runs the per-layer kernel's own per-pair code, so sites, bonds,
  norm_log, kept counts, spectra and statuses are bit-identical to launching
  the layers one by one with the same kernel shape (the "split" strategy:
  one launch per bond-cap class and layer) -- checked on uneven chains of every bond-cap class
  (16 / 32 / 64: all three CTA shapes, and the tensor-core form at 64), for
  every CTA size the autotuner may pick.
* A dependency wait that runs out is reported, not hung on: with a poll limit
  of 0 an update whose predecessor (a saturated chi = 64 pair, ~1 ms) is still
  running gives up at once, is skipped with MPSB_ST_TIMEOUT, the launch
  returns, and the device stays usable.
"""
import numpy as np
import pytest
import torch

from fpga_mps_simulator_b200.circuits import brickwall_layers, random_circuit_batch

pytestmark = pytest.mark.gpu


def _specs(chis):
    return random_circuit_batch(9, seed=5, n_range=(8, 30), depth_range=(4, 12), chis=chis)


def _run_both(specs, precision, threads):
    from fpga_mps_simulator_b200 import MPSBatch
    from fpga_mps_simulator_b200.schedule import Runner, Schedule
    out = []
    for strategy in ("split", "flow"):  # both launch each bond-cap class with its own cap
        b = MPSBatch([s.n for s in specs], [s.chi_max for s in specs], 1e-10, precision=precision)
        sch = Schedule(b, [s.layers for s in specs], record_spectra=True)
        if strategy == "flow":
            sch.flow_threads.update(threads)
        Runner(sch, strategy).run()
        torch.cuda.synchronize()
        b.check_status()
        out.append((b, sch))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("threads", [{}, {16: 128, 32: 256}])
def test_flow_is_bitwise_the_per_layer_result(precision, threads):
    specs = _specs((16, 32, 64))
    (bl, sl), (bf, sf) = _run_both(specs, precision, threads)
    for x, y in zip(bl.snapshot(), bf.snapshot()):
        assert torch.equal(x, y)
    # per-update outputs: the flow lists each class's updates layer by layer
    # in the per-layer tables' order, so the rows line up after regrouping
    per_layer = {}
    for ls in sl.launches("split"):
        for lc in ls:
            pr = lc.pb.pairs.cpu().numpy()
            for row, (c, i) in enumerate(pr[:, :2]):
                per_layer.setdefault((int(c), int(i)), []).append(
                    (int(lc.pb.kept[row]), lc.pb.spectra[row].cpu().numpy(), int(lc.pb.status[row])))
    for fl in sf.flow_plan():
        items = fl.fb.host_items
        kept, spec, st = fl.fb.kept.cpu().numpy(), fl.fb.spectra.cpu().numpy(), fl.fb.status.cpu().numpy()
        for k, (c, i) in enumerate(items[:, :2]):
            kk, ss, tt = per_layer[(int(c), int(i))].pop(0)
            assert kk == kept[k] and tt == st[k] == 0
            assert np.array_equal(ss, spec[k])
    assert all(not v for v in per_layer.values())


def test_dependency_wait_that_runs_out_is_reported_and_the_device_stays_usable():
    from fpga_mps_simulator_b200 import MPSBatch, _lib
    n, chi = 20, 64
    layers = brickwall_layers(n, 10, 31)
    b = MPSBatch([n], [chi], 1e-10)
    for L in layers[:8]:  # saturate the middle bonds: a chi = 64 pair takes ~1 ms
        b.apply_layer(np.zeros(len(L.sites), np.int32), L.sites, L.gates)
    torch.cuda.synchronize()
    assert b.bond_dims(0)[9] == chi
    before = b.snapshot()
    g = layers[8].gates
    fb = b.make_flow([0, 0], [9, 10], g[:2])  # item 1 (sites 10, 11) waits for item 0 (sites 9, 10)
    assert fb.host_items[1, 4] == 0
    b.run_flow(fb, poll_limit=0)
    torch.cuda.synchronize()
    st = fb.status.cpu().numpy()
    assert st[0] == 0 and st[1] == _lib.ST_TIMEOUT
    assert int(b.check_status(raise_on_error=False)[0]) & _lib.ST_TIMEOUT
    # the skipped update left its second site alone; the first update happened
    k = int(b.bond_off[0])
    assert torch.equal(b.sites[k + 11], before[0][k + 11])
    assert not torch.equal(b.sites[k + 9], before[0][k + 9])
    # the context is intact: the same two updates with the default limit match per-layer launches
    b.restore(before)
    b.status_acc.zero_()
    fb2 = b.make_flow([0, 0], [9, 10], g[:2])
    b.run_flow(fb2)
    ref = MPSBatch([n], [chi], 1e-10)
    ref.restore(before)
    ref.status_acc.zero_()
    ref.apply_layer([0], [9], g[:1])
    ref.apply_layer([0], [10], g[1:2])
    torch.cuda.synchronize()
    b.check_status()
    ref.check_status()
    for x, y in zip(b.snapshot(), ref.snapshot()):
        assert torch.equal(x, y)
