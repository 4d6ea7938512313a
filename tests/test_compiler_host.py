"""Circuit compiler on the host (no GPU): the gate list equals the reference
compiler's (fpga_mps_simulator.py:285-410) on the golden circuits, and the
layer schedule (single-site fusion, as-soon-as-possible layers) is the same
unitary as the gate list it came from."""
import numpy as np
import pytest

from conftest import load_golden
from oracle.mps_oracle import dense_apply_1q, dense_apply_2q, dense_zero_state
from fpga_mps_simulator_b200.compiler import Circuit, compile_circuit, schedule


def golden_circuits():
    g = load_golden("compiler")
    out = []
    for idx in range(int(g["count"])):
        p = f"c{idx}_"
        n = int(g[p + "n"])
        c = Circuit(n)
        for nm, qs, ps, k in zip(g[p + "ins_names"], g[p + "ins_qubits"], g[p + "ins_params"], g[p + "ins_nparams"]):
            c.append(str(nm), [int(q) for q in qs if q >= 0], list(ps[:k]))
        out.append((c, g, p))
    return out


@pytest.mark.parametrize("idx", range(12))
def test_gate_list_matches_reference_compiler(idx):
    c, g, p = golden_circuits()[idx]
    gl, meas = compile_circuit(c, c.num_qubits)
    assert meas == list(g[p + "measured"])
    assert [x["type"] for x in gl] == list(g[p + "gl_type"])
    assert [x["gate_name"] for x in gl] == list(g[p + "gl_name"])
    for x, sites, mat in zip(gl, g[p + "gl_sites"], g[p + "gl_mat"]):
        assert x["sites"] == [int(s) for s in sites if s >= 0]
        if x["gate_mat"] is not None:
            m = np.asarray(x["gate_mat"]).reshape(-1)
            np.testing.assert_allclose(m, mat[:m.size], atol=1e-15)


def _dense_run_gates(gl, n):
    psi = dense_zero_state(n)
    for x in gl:
        if x["type"] == "1q":
            psi = dense_apply_1q(psi, x["sites"][0], x["gate_mat"])
        elif x["type"] == "2q":
            psi = dense_apply_2q(psi, x["sites"][0], x["sites"][1], x["gate_mat"])
        else:
            return None
    return psi


def _dense_run_program(prog, n):
    psi = dense_zero_state(n)
    for L in prog.layers:
        if L["reset"]:
            return None
        for s, gm in L["one"]:
            psi = dense_apply_1q(psi, s, gm)
        for i, gm in L["two"]:
            psi = dense_apply_2q(psi, i, i + 1, gm)
    return psi


def _random_unitary_circuits(count=10):
    out = []
    for seed in range(count):
        rng = np.random.default_rng(500 + seed)
        n = int(rng.integers(3, 8))
        c = Circuit(n)
        for _ in range(40):
            k = int(rng.integers(0, 5))
            if k < 2:
                c.append(str(rng.choice(["h", "t", "sx", "y"])), [int(rng.integers(n))])
            elif k == 2:
                c.append("u", [int(rng.integers(n))], list(rng.uniform(-3, 3, 3)))
            elif k == 3:
                a, b = rng.choice(n, 2, replace=False)
                c.append(str(rng.choice(["cx", "rzz", "iswap", "ecr"])), [int(a), int(b)], [0.4])
            else:
                a, b, t = rng.choice(n, 3, replace=False)
                c.append("ccx", [int(a), int(b), int(t)])
        out.append(c)
    return out


@pytest.mark.parametrize("fuse", [True, False])
def test_schedule_is_the_same_unitary(fuse):
    checked = 0
    for c in [x[0] for x in golden_circuits()] + _random_unitary_circuits():
        gl, _ = compile_circuit(c, c.num_qubits)
        if any(x["type"] == "reset" for x in gl):
            continue
        prog = schedule(gl, c.num_qubits, fuse)
        for L in prog.layers:   # disjoint sites inside a layer
            used = [s for s, _ in L["one"]] + L["reset"] + [s for i, _ in L["two"] for s in (i, i + 1)]
            assert len(used) == len(set(used))
        a, b = _dense_run_gates(gl, c.num_qubits), _dense_run_program(prog, c.num_qubits)
        np.testing.assert_allclose(b, a, atol=1e-12)
        checked += 1
    assert checked >= 10


def test_fusion_removes_single_site_launches():
    c = Circuit(4)
    for q in range(4):
        c.h(q)
        c.rz(q, 0.3)
    c.cx(0, 1)
    c.cx(2, 3)
    c.cx(1, 2)
    gl, _ = compile_circuit(c, 4)
    prog = schedule(gl, 4)
    assert prog.counts() == {"one": 0, "reset": 0, "two": 3}
    assert prog.depth == 2


def test_unsupported_instruction_raises():
    c = Circuit(2)
    c.append("mystery", [0])
    with pytest.raises(ValueError):
        compile_circuit(c, 2)
