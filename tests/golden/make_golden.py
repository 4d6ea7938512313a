"""Generate the golden fixtures in this folder by running the reference engine.

Run from the repository root with a checkout of the reference repository,
given as the first argument or in the environment variable MPS_REFERENCE_DIR:

    python tests/golden/make_golden.py /path/to/reference [run_NAME ...]

It imports the reference's ``mps_core.py`` unchanged, drives it through its own
public methods (``apply_1q``, ``apply_2q``, ``_apply_adjacent_2q``,
``get_statevector``, ``get_counts``) and records what they return.  The
per-update singular values are captured by wrapping ``la.svd`` inside the
reference module, which leaves its numerics untouched.  Circuits come from the
reference's own checks: the six small circuits of ``fpga_diag.py:28-58`` and
the 3-qubit GHZ self-test of ``fpga_mps_simulator.py:1147-1165``, re-expressed
as gate-list calls because Qiskit is not installed.

The committed ``.npz`` files are what the tests read; this script is not run
by the tests.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ARGS = [a for a in sys.argv[1:] if not a.startswith("--")]
REF = _ARGS[0] if _ARGS and not _ARGS[0].startswith("run_") else os.environ.get("MPS_REFERENCE_DIR", "")
if not REF or not os.path.isfile(os.path.join(REF, "mps_core.py")):
    sys.exit("make_golden.py: give the reference checkout (the folder holding mps_core.py) as the first "
             "argument or in MPS_REFERENCE_DIR")
sys.path.insert(0, REF)
import mps_core  # noqa: E402  (the reference module, unchanged)


def haar(rng):
    z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def brick(n, depth, seed):
    rng = np.random.default_rng(seed)
    out = []
    for layer in range(depth):
        for i in range(layer % 2, n - 1, 2):
            out.append((i, haar(rng)))
    return out


class Recorder:
    """Wrap the reference module's SVD call to capture every spectrum."""

    def __init__(self):
        self.spectra = []
        self._orig = mps_core.la.svd

    def __enter__(self):
        def svd(*a, **k):
            u, s, vh = self._orig(*a, **k)
            self.spectra.append(np.array(s, copy=True))
            return u, s, vh
        mps_core.la.svd = svd
        return self

    def __exit__(self, *exc):
        mps_core.la.svd = self._orig


def pack_spectra(spectra):
    width = max(len(s) for s in spectra)
    arr = np.zeros((len(spectra), width))
    lens = np.zeros(len(spectra), dtype=np.int32)
    for k, s in enumerate(spectra):
        arr[k, :len(s)] = s
        lens[k] = len(s)
    return arr, lens


def amplitudes(st, bit_rows):
    out = []
    for bits in bit_rows:
        v = np.ones((1,), np.complex128)
        for k in range(st.n):
            v = v @ st.sites[k][:, int(bits[k]), :]
        out.append(v[0] * math.exp(st.norm_log))
    return np.array(out)


def run_brick(name, n, depth, chi, cutoff, seed, n_amp=64, full_sv=False):
    gates = brick(n, depth, seed)
    st = mps_core.MPSState(n, chi, cutoff)
    norm_logs, bonds = [], []
    with Recorder() as rec:
        for i, g in gates:
            st._apply_adjacent_2q(i, g)
            norm_logs.append(st.norm_log)
            bonds.append(st.bond_dims())
    spec, lens = pack_spectra(rec.spectra)
    rng = np.random.default_rng(seed + 1)
    bit_rows = rng.integers(0, 2, size=(n_amp, n))
    bit_rows[0] = 0
    data = dict(n=n, depth=depth, chi_max=chi, cutoff=cutoff, seed=seed,
                sites=np.array([i for i, _ in gates], np.int32),
                gates=np.stack([g for _, g in gates]),
                spectra=spec, spec_len=lens, norm_log=np.array(norm_logs),
                bonds=np.array(bonds, np.int32), bits=bit_rows.astype(np.int8),
                amps=amplitudes(st, bit_rows))
    if full_sv:
        data["statevector"] = st.get_statevector()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
    print(name, "updates", len(gates), "max bond", st.max_bond(), "norm_log", st.norm_log)


def run_gate_tables():
    names_1q = sorted(mps_core._SINGLE_QUBIT_GATES)
    names_2q = sorted(mps_core._TWO_QUBIT_GATES - {"cnot"})
    params = [0.37, -1.21, 2.05]
    g1 = np.stack([mps_core._gate_1q(nm, params) for nm in names_1q])
    g2 = np.stack([mps_core._gate_2q(nm, params) for nm in names_2q])
    np.savez_compressed(os.path.join(HERE, "gate_tables.npz"),
                        names_1q=np.array(names_1q), names_2q=np.array(names_2q),
                        params=np.array(params), g1=g1, g2=g2)


def run_diag_circuits():
    """fpga_diag.py:28-58 as mps_core gate-list calls, plus the GHZ-3 self-test."""
    U = mps_core._gate_1q
    G2 = mps_core._gate_2q
    cases = {
        "bell": (2, [("1", 0, U("h", None)), ("2", 0, 1, G2("cx", None))]),
        "ghz4": (4, [("1", 0, U("h", None))] + [("2", i, i + 1, G2("cx", None)) for i in range(3)]),
        "cx03": (4, [("1", 0, U("h", None)), ("2", 0, 3, G2("cx", None))]),
        "u1": (1, [("1", 0, U("u", [0.7, 1.3, -0.4]))]),
        "ucxu": (2, [("1", 0, U("u", [0.7, 1.3, -0.4])), ("1", 1, U("u", [-0.9, 0.2, 2.1])),
                     ("2", 0, 1, G2("cx", None)), ("1", 0, U("u", [0.3, -0.6, 1.1]))]),
        "ucx02": (4, [("1", 0, U("u", [0.7, 1.3, -0.4])), ("1", 2, U("u", [-0.9, 0.2, 2.1])),
                      ("2", 0, 2, G2("cx", None))]),
        "ghz3": (3, [("1", 0, U("h", None)), ("2", 0, 1, G2("cx", None)), ("2", 1, 2, G2("cx", None))]),
    }
    out = {}
    for key, (n, ops) in cases.items():
        st = mps_core.MPSState(n, 64, 1e-12)
        enc = []
        for op in ops:
            if op[0] == "1":
                st.apply_1q(op[1], op[2])
                enc.append((1, op[1], -1, np.pad(op[2].reshape(-1), (0, 12))))
            else:
                st.apply_2q(op[1], op[2], op[3])
                enc.append((2, op[1], op[2], op[3].reshape(-1)))
        out[key + "_n"] = n
        out[key + "_kind"] = np.array([e[0] for e in enc], np.int32)
        out[key + "_qa"] = np.array([e[1] for e in enc], np.int32)
        out[key + "_qb"] = np.array([e[2] for e in enc], np.int32)
        out[key + "_mat"] = np.stack([e[3] for e in enc])
        out[key + "_sv"] = st.get_statevector()
        if key == "ghz3":
            counts = st.get_counts(1024, rng=np.random.default_rng(0))
            out["ghz3_count_keys"] = np.array(sorted(counts))
            out["ghz3_count_vals"] = np.array([counts[k] for k in sorted(counts)], np.int64)
    np.savez_compressed(os.path.join(HERE, "diag_circuits.npz"), **out)


def run_xxz():
    """Low-entanglement case: random product state + XXZ second-order Trotter."""
    import scipy.linalg as sla
    n, steps, dt, chi, cutoff, seed = 24, 6, 0.05, 16, 1e-10, 5
    x = np.array([[0, 1], [1, 0]], complex)
    y = np.array([[0, -1j], [1j, 0]])
    z = np.diag([1.0, -1.0]).astype(complex)
    h = np.kron(x, x) + np.kron(y, y) + 0.5 * np.kron(z, z)
    half, full = sla.expm(-0.5j * dt * h), sla.expm(-1j * dt * h)
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    st = mps_core.MPSState(n, chi, cutoff)
    for i in range(n):
        st.apply_1q(i, mps_core._gate_1q("u", [th[i], ph[i], 0.0]))
    seq = []
    for _ in range(steps):
        seq += [(i, half) for i in range(1, n - 1, 2)]
        seq += [(i, full) for i in range(0, n - 1, 2)]
        seq += [(i, half) for i in range(1, n - 1, 2)]
    norm_logs = []
    with Recorder() as rec:
        for i, g in seq:
            st._apply_adjacent_2q(i, g)
            norm_logs.append(st.norm_log)
    spec, lens = pack_spectra(rec.spectra)
    bit_rows = np.random.default_rng(seed + 1).integers(0, 2, size=(32, n))
    np.savez_compressed(os.path.join(HERE, "xxz.npz"), n=n, chi_max=chi, cutoff=cutoff,
                        theta=th, phi=ph, sites=np.array([i for i, _ in seq], np.int32),
                        gates=np.stack([g for _, g in seq]), spectra=spec, spec_len=lens,
                        norm_log=np.array(norm_logs), bits=bit_rows.astype(np.int8),
                        amps=amplitudes(st, bit_rows), bonds=np.array(st.bond_dims(), np.int32))
    print("xxz max bond", st.max_bond(), "norm_log", st.norm_log)


def pack_sites(sites):
    shapes = np.array([t.shape for t in sites], np.int32)
    flat = np.concatenate([t.reshape(-1) for t in sites])
    return shapes, flat


def run_measure():
    """Shots of MPSState.sample / get_counts and the canonical-form helpers
    (left/right_normalize_site sweeps, entanglement_entropy, bond_spectrum)."""
    n, depth, chi, cutoff, seed = 16, 10, 16, 1e-12, 1234
    st = mps_core.MPSState(n, chi, cutoff)
    for i, g in brick(n, depth, seed):
        st._apply_adjacent_2q(i, g)
    shots = st.sample(400, rng=np.random.default_rng(11))
    sub_q = [0, 3, 7, 12]
    sub = st.sample(200, measured_qubits=sub_q, rng=np.random.default_rng(12))
    counts = st.get_counts(300, rng=np.random.default_rng(13))
    # canonical forms of a random, non-canonical chain
    rng = np.random.default_rng(21)
    bonds = [1, 2, 4, 8, 6, 5, 3, 2, 1]
    m = len(bonds) - 1
    sites = [(rng.standard_normal((bonds[k], 2, bonds[k + 1]))
              + 1j * rng.standard_normal((bonds[k], 2, bonds[k + 1]))) for k in range(m)]
    ref = mps_core.MPSState(m, 64, 1e-12)
    ref.sites = [t.copy() for t in sites]
    ent = np.array([ref.entanglement_entropy(b) for b in range(m - 1)])
    spec = [ref.bond_spectrum(b) for b in range(m - 1)]
    left = ref.copy()
    left.left_canonicalize()
    right = ref.copy()
    right.right_canonicalize()
    in_shapes, in_flat = pack_sites(sites)
    l_shapes, l_flat = pack_sites(left.sites)
    r_shapes, r_flat = pack_sites(right.sites)
    sp_len = np.array([len(x) for x in spec], np.int32)
    sp = np.zeros((len(spec), sp_len.max()))
    for k, x in enumerate(spec):
        sp[k, :len(x)] = x
    np.savez_compressed(os.path.join(HERE, "measure.npz"), n=n, depth=depth, chi_max=chi, cutoff=cutoff,
                        seed=seed, shots=np.array(shots), sub_qubits=np.array(sub_q, np.int32),
                        sub_shots=np.array(sub), count_keys=np.array(sorted(counts)),
                        count_vals=np.array([counts[k] for k in sorted(counts)], np.int64),
                        canon_in_shapes=in_shapes, canon_in=in_flat, left_shapes=l_shapes, left=l_flat,
                        right_shapes=r_shapes, right=r_flat, entropy=ent, bond_spectrum=sp,
                        bond_spectrum_len=sp_len)
    print("measure: shots", len(shots), "distinct", len(set(shots)))


def run_dropin():
    """What a drop-in user of the reference class sees: entanglement_entropy and
    bond_spectrum (mps_core.py:465-494) on every bond of two circuit states, and
    the default bond cap (MPSState(n) keeps chi_max=256, mps_core.py:185): a
    12-qubit circuit whose bonds stay within 64, and a 14-qubit one whose
    middle bond needs 128."""
    out = {}
    for key, (n, depth, chi, cutoff, seed) in {"b16": (16, 10, 16, 1e-12, 1234),
                                                "b20": (20, 12, 64, 1e-10, 4242)}.items():
        st = mps_core.MPSState(n, chi, cutoff)
        for i, g in brick(n, depth, seed):
            st._apply_adjacent_2q(i, g)
        spec = [st.bond_spectrum(b) for b in range(n)]
        lens = np.array([len(x) for x in spec], np.int32)
        sp = np.zeros((n, lens.max()))
        for k, x in enumerate(spec):
            sp[k, :len(x)] = x
        out[key + "_entropy"] = np.array([st.entanglement_entropy(b) for b in range(n - 1)])
        out[key + "_bond_spectrum"] = sp
        out[key + "_bond_spectrum_len"] = lens
        out[key + "_bonds"] = np.array(st.bond_dims(), np.int32)
    for key, (n, depth, seed) in {"d12": (12, 10, 99), "d14": (14, 12, 98)}.items():
        st = mps_core.MPSState(n)
        gates = brick(n, depth, seed)
        for i, g in gates:
            st._apply_adjacent_2q(i, g)
        bits = np.random.default_rng(seed + 1).integers(0, 2, size=(32, n))
        out[key + "_chi_max"] = st.chi_max
        out[key + "_cutoff"] = st.svd_cutoff
        out[key + "_sites"] = np.array([i for i, _ in gates], np.int32)
        out[key + "_gates"] = np.stack([g for _, g in gates])
        out[key + "_bonds"] = np.array(st.bond_dims(), np.int32)
        out[key + "_norm_log"] = st.norm_log
        out[key + "_bits"] = bits.astype(np.int8)
        out[key + "_amps"] = amplitudes(st, bits)
    np.savez_compressed(os.path.join(HERE, "dropin.npz"), **out)
    print("dropin: max bonds", out["d12_bonds"].max(), out["d14_bonds"].max())


class _Q:
    def __init__(self, i):
        self.index = i


class _Inst:
    def __init__(self, name, qubits, params):
        self.operation = type("Op", (), {"name": name, "params": list(params)})()
        self.qubits = qubits


class DuckCircuit:
    """The attribute shape of qiskit's QuantumCircuit that compile_circuit reads."""

    def __init__(self, n):
        self.num_qubits = n
        self.qubits = [_Q(i) for i in range(n)]
        self.data = []

    def find_bit(self, q):
        return type("Loc", (), {"index": q.index})()

    def add(self, name, qs, params=()):
        self.data.append(_Inst(name, [self.qubits[q] for q in qs], params))


def random_instructions(seed):
    """Seeded random instruction list (name, qubits, params) over 3..9 qubits."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 10))
    out = []
    for _ in range(int(rng.integers(10, 40))):
        k = int(rng.integers(0, 7))
        if k < 2:
            out.append((str(rng.choice(["h", "x", "t", "sdg", "sx", "y"])), [int(rng.integers(n))], []))
        elif k == 2:
            out.append(("u", [int(rng.integers(n))], [float(v) for v in rng.uniform(-3, 3, 3)]))
        elif k in (3, 4):
            a, b = rng.choice(n, 2, replace=False)
            nm = str(rng.choice(["cx", "cz", "rzz", "swap", "cp", "ecr", "iswap", "rxx"]))
            out.append((nm, [int(a), int(b)], [0.37] if nm in ("rzz", "cp", "rxx") else []))
        elif k == 5:
            a, b, t = rng.choice(n, 3, replace=False)
            out.append(("ccx", [int(a), int(b), int(t)], []))
        else:
            out.append(("measure" if rng.random() < 0.6 else "reset", [int(rng.integers(n))], []))
    return n, out


def run_compiler():
    """Reference compile_circuit on seeded random circuits, then the gate list
    executed by the reference engine (MPSState for the gates, the reset branch of
    _run_circuit_fpga restated, get_counts with default_rng(seed + index))."""
    import fpga_mps_simulator as fms  # the reference execution engine module, unchanged
    out = {}
    base_seed, shots = 100, 256
    for idx in range(12):
        n, ins = random_instructions(1000 + idx)
        c = DuckCircuit(n)
        for nm, qs, ps in ins:
            c.add(nm, qs, ps)
        gl, meas = fms.compile_circuit(c, n)
        st = mps_core.MPSState(n, 64, 1e-12)
        for g in gl:
            if g["type"] == "1q":
                st.apply_1q(g["sites"][0], g["gate_mat"])
            elif g["type"] == "2q":
                st._apply_adjacent_2q(g["sites"][0], g["gate_mat"])
            else:
                s = g["sites"][0]
                t = st.sites[s].copy()
                t[:, 1, :] = 0.0
                nm = np.linalg.norm(t)
                if nm > 1e-15:
                    t /= nm
                else:
                    t = np.zeros_like(t)
                    t[0, 0, 0] = 1.0
                st.sites[s] = t
        counts = st.get_counts(shots, meas, np.random.default_rng(base_seed + idx))
        p = f"c{idx}_"
        out[p + "n"] = n
        out[p + "ins_names"] = np.array([i[0] for i in ins])
        out[p + "ins_qubits"] = np.array([i[1] + [-1] * (3 - len(i[1])) for i in ins], np.int32)
        out[p + "ins_params"] = np.array([i[2] + [0.0] * (3 - len(i[2])) for i in ins])
        out[p + "ins_nparams"] = np.array([len(i[2]) for i in ins], np.int32)
        out[p + "gl_type"] = np.array([g["type"] for g in gl])
        out[p + "gl_name"] = np.array([g["gate_name"] for g in gl])
        out[p + "gl_sites"] = np.array([g["sites"] + [-1] * (2 - len(g["sites"])) for g in gl], np.int32)
        out[p + "gl_mat"] = np.stack([np.zeros(16, complex) if g["gate_mat"] is None
                                      else np.pad(np.asarray(g["gate_mat"]).reshape(-1), (0, 16 - g["gate_mat"].size))
                                      for g in gl])
        out[p + "measured"] = np.array(meas, np.int32)
        out[p + "sv"] = st.get_statevector()
        out[p + "count_keys"] = np.array(sorted(counts))
        out[p + "count_vals"] = np.array([counts[k] for k in sorted(counts)], np.int64)
    out["count"] = 12
    out["shots"] = shots
    out["seed"] = base_seed
    np.savez_compressed(os.path.join(HERE, "compiler.npz"), **out)
    print("compiler: 12 circuits")


RUNS = {
    "run_gate_tables": run_gate_tables,
    "run_diag_circuits": run_diag_circuits,
    "run_brick_n16": lambda: run_brick("brick_n16_d10_chi16", 16, 10, 16, 1e-12, 1234, full_sv=True),
    "run_brick_n40": lambda: run_brick("brick_n40_d16_chi32", 40, 16, 32, 1e-10, 77),
    "run_brick_n20": lambda: run_brick("brick_n20_d12_chi64", 20, 12, 64, 1e-10, 4242),
    "run_xxz": run_xxz,
    "run_measure": run_measure,
    "run_compiler": run_compiler,
    "run_dropin": run_dropin,
}

if __name__ == "__main__":
    only = [a for a in sys.argv[1:] if a.startswith("run_")]
    for name, fn in RUNS.items():
        if not only or name in only:
            fn()
