"""Hand-written adjoint of circuits of two-site updates and single-site gates.

The reference engine (mps_core.py of nasir26/fpga-mps-simulator) has no
gradients.  This module differentiates exactly what the device forward
computes -- contract, gate, truncated SVD (keep rule and renormalisation of
mps_core.py:277-300), sqrt(S) split -- for the normalised energy
L = <psi|H|psi> / <psi|psi> of a matrix-product operator H, with the device
kernels of libmpsb200:

* ``mpsb_mpo_energy_grad``: L and the cotangent of every final site;
* ``mpsb_update2q_backward_batch``: one layer of two-site updates, from the
  tape a taped forward of that layer recorded (truncated-SVD backward with
  the kept/discarded coupling and Lorentzian-broadened 1/(s_j^2 - s_i^2));
* ``mpsb_apply1q_backward_batch``: one layer of single-site gates, with the
  gate cotangents from which the angle gradients follow.

Checkpointing: the forward keeps only the state at the start of every group
of steps (one ansatz layer, one Trotter step); the backward restores each
checkpoint in turn, recomputes that group with tapes (bit-identical to the
forward: same kernels, same inputs) and runs its backward.  With
``checkpoint=False`` every step keeps its tape and saved input from the
forward instead (no recomputation, more memory); ``checkpoint="auto"``
(the default) does that whenever the whole program's tapes fit in half of
the device memory that is free when the forward starts.

``HEAEnergy`` is config "differentiation" (RY, RZ on every site, CZ on
brick-wall pairs, transverse-field Ising energy, many parameter vectors as
independent chains of one batch) and ``HEAEnergyFunction`` wraps it as a
``torch.autograd.Function``.  ``XXZInitialStateGradient`` differentiates a
Trotterised XXZ evolution with respect to the Bloch angles of the initial
product state.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from .circuits import Layer, xxz_trotter_layers
from .hamiltonians import check_mpo, tfim_mpo, zz_mpo
from .mps import PRECISIONS, MPSBatch, PairBatch, _Workspace

__all__ = ["Step1Q", "Step2Q", "AdjointEngine", "HEAEnergy", "HEAEnergyFunction", "XXZInitialStateGradient",
           "rot_gates", "rot_angle_grads"]

_CZ = np.diag([1, 1, 1, -1]).astype(np.complex128)


@dataclass
class Step1Q:
    """Single-site gates: ops (nops, 4) int32 device rows (chain, site, gate, 0) on
    distinct sites; gates (nops, 2, 2) complex128 device (set before each run)."""
    ops: torch.Tensor
    gates: torch.Tensor
    key: str


@dataclass
class Step2Q:
    """One launch of disjoint two-site updates with fixed gates."""
    pb: PairBatch
    chi_cap: int


Step = Union[Step1Q, Step2Q]


class AdjointEngine:
    """Forward with checkpoints and hand-written backward over groups of steps."""

    def __init__(self, batch: MPSBatch, mpo: np.ndarray, checkpoint: Union[bool, str] = "auto"):
        if len(set(batch.ns)) != 1:
            raise ValueError("the energy gradient needs chains of equal length")
        self.b = batch
        self.lib = _lib.OnDevice(_lib.load(), batch.device)
        self.n = batch.ns[0]
        W = check_mpo(mpo, self.n)
        self.D = W.shape[1]
        self.mpo = torch.from_numpy(W.reshape(-1)).to(batch.device)
        if checkpoint not in (True, False, "auto"):
            raise ValueError("checkpoint must be True, False or 'auto'")
        self.checkpoint = checkpoint
        self.checkpointed = checkpoint is True
        self.cot = torch.zeros_like(batch.sites)
        self.cot_table = batch.make_table(self.cot, batch.bonds)
        self.loss = torch.zeros(batch.nchains, dtype=torch.float64, device=batch.device)
        self._ws_fwd = _Workspace(batch.device)
        self._ws_bwd = _Workspace(batch.device)
        self._ws_loss = _Workspace(batch.device)
        self.groups: List[List[Step]] = []
        self.ckpts: List[Tuple[torch.Tensor, torch.Tensor]] = []
        self.records: List[list] = []
        self.final: Optional[Tuple[torch.Tensor, torch.Tensor]] = None
        self.launches = 0

    # -- one step ----------------------------------------------------------------
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.b.device).cuda_stream

    def _run(self, step: Step, tape: Optional[torch.Tensor] = None) -> None:
        b = self.b
        if isinstance(step, Step1Q):
            rc = self.lib.mpsb_apply1q_batch(b.table.data_ptr(), step.ops.data_ptr(), step.ops.shape[0],
                                             step.gates.data_ptr(), b.chi_cap, self._stream())
            _lib.check(rc, "mpsb_apply1q_batch")
            self.launches += 1
            return
        pb = step.pb
        if tape is None:
            b.run_pairs(pb, chi_cap=step.chi_cap)
            self.launches += 2
            return
        need = self.lib.mpsb_update2q_workspace_bytes(pb.npairs, step.chi_cap)
        ws = self._ws_fwd.get(need)
        rc = self.lib.mpsb_update2q_batch_taped(
            b.table.data_ptr(), pb.pairs.data_ptr(), pb.npairs, pb.gates.data_ptr(), PRECISIONS[b.precision],
            step.chi_cap, b.tol, b.max_sweeps, ws.data_ptr(), ws.numel(), tape.data_ptr(), tape.numel(),
            None, pb.kept.data_ptr(), pb.trunc.data_ptr(), pb.status.data_ptr(), self._stream())
        _lib.check(rc, "mpsb_update2q_batch_taped")
        self.launches += 2

    def _record(self, step: Step) -> tuple:
        """Run one step keeping what its backward needs: its input state and (2q) its tape."""
        b = self.b
        pre = (b.sites.clone(), b.bonds.clone())
        tape = None
        if isinstance(step, Step2Q):
            nbytes = self.lib.mpsb_update2q_tape_bytes(step.pb.npairs, step.chi_cap)
            tape = torch.empty(nbytes, dtype=torch.uint8, device=b.device)
        self._run(step, tape)
        return (step, pre, tape)

    def _backward_step(self, rec: tuple, grads: Dict[str, torch.Tensor]) -> None:
        step, (pre_sites, pre_bonds), tape = rec
        b = self.b
        pre_table = b.make_table(pre_sites, pre_bonds)
        if isinstance(step, Step1Q):
            gg = torch.empty(step.ops.shape[0], 4, dtype=torch.complex128, device=b.device)
            rc = self.lib.mpsb_apply1q_backward_batch(pre_table.data_ptr(), self.cot_table.data_ptr(),
                                                      step.ops.data_ptr(), step.ops.shape[0], step.gates.data_ptr(),
                                                      b.chi_cap, gg.data_ptr(), self._stream())
            _lib.check(rc, "mpsb_apply1q_backward_batch")
            grads[step.key] = gg.reshape(-1, 2, 2)
        else:
            pb = step.pb
            need = self.lib.mpsb_update2q_backward_workspace_bytes(pb.npairs, step.chi_cap)
            ws = self._ws_bwd.get(need)
            status = torch.zeros(pb.npairs, dtype=torch.int32, device=b.device)
            rc = self.lib.mpsb_update2q_backward_batch(
                pre_table.data_ptr(), self.cot_table.data_ptr(), pb.pairs.data_ptr(), pb.npairs, pb.gates.data_ptr(),
                step.chi_cap, tape.data_ptr(), tape.numel(), None, ws.data_ptr(), ws.numel(), status.data_ptr(),
                self._stream())
            _lib.check(rc, "mpsb_update2q_backward_batch")
            self._bwd_status.append(status)
        self.launches += 1

    # -- whole program ---------------------------------------------------------------
    def tape_bytes(self, groups: Sequence[Sequence[Step]]) -> int:
        """Device bytes a forward that keeps every step's tape and input would hold."""
        b = self.b
        state = b.sites.numel() * b.sites.element_size() + b.bonds.numel() * 4
        total = 0
        for g in groups:
            for st in g:
                total += state
                if isinstance(st, Step2Q):
                    total += self.lib.mpsb_update2q_tape_bytes(st.pb.npairs, st.chi_cap)
        return total

    def forward(self, groups: Sequence[Sequence[Step]]) -> None:
        """Run the program from the batch's current state, keeping checkpoints (or tapes)."""
        b = self.b
        self.groups = [list(g) for g in groups]
        self.ckpts, self.records = [], []
        if self.checkpoint == "auto":
            free, _ = torch.cuda.mem_get_info(b.device)
            self.checkpointed = self.tape_bytes(self.groups) > free // 2
        else:
            self.checkpointed = bool(self.checkpoint)
        for g in self.groups:
            if self.checkpointed:
                self.ckpts.append((b.sites.clone(), b.bonds.clone()))
                for st in g:
                    self._run(st)
            else:
                self.records.append([self._record(st) for st in g])
        self.final = (b.sites.clone(), b.bonds.clone())

    def energy(self, weights: Optional[torch.Tensor] = None) -> torch.Tensor:
        """L per chain for the current state; also writes the cotangent of every site."""
        b = self.b
        need = self.lib.mpsb_mpo_grad_workspace_bytes(b.nchains, self.n, b.chi_cap, self.D)
        ws = self._ws_loss.get(need)
        self.cot.zero_()
        rc = self.lib.mpsb_mpo_energy_grad(b.table.data_ptr(), b.nchains, self.n, b.chi_cap, self.mpo.data_ptr(),
                                           self.D, None if weights is None else weights.data_ptr(),
                                           self.loss.data_ptr(), self.cot_table.data_ptr(), ws.data_ptr(),
                                           ws.numel(), self._stream())
        _lib.check(rc, "mpsb_mpo_energy_grad")
        self.launches += 2
        return self.loss

    def backward(self, weights: Optional[torch.Tensor] = None) -> Dict[str, torch.Tensor]:
        """Cotangents of every Step1Q's gates (by key); self.cot ends as the
        cotangent of the state the forward started from.  The batch is left in
        the forward's final state."""
        b = self.b
        if self.final is None:
            raise RuntimeError("backward() needs a forward() first")
        b.sites.copy_(self.final[0])
        b.bonds.copy_(self.final[1])
        if weights is not None:
            weights = weights.to(device=b.device, dtype=torch.float64).contiguous()
        self.energy(weights)
        grads: Dict[str, torch.Tensor] = {}
        self._bwd_status: List[torch.Tensor] = []
        for gi in range(len(self.groups) - 1, -1, -1):
            if self.checkpointed:
                b.sites.copy_(self.ckpts[gi][0])
                b.bonds.copy_(self.ckpts[gi][1])
                recs = [self._record(st) for st in self.groups[gi]]
            else:
                recs = self.records[gi]
            for rec in reversed(recs):
                self._backward_step(rec, grads)
            del recs
            if not self.checkpointed:
                self.records[gi] = None  # release this group's tapes as soon as they are used
        b.sites.copy_(self.final[0])
        b.bonds.copy_(self.final[1])
        if self._bwd_status:
            st = torch.cat(self._bwd_status)
            if bool((st != 0).any()):
                raise RuntimeError(f"two-site backward reported status bits {int(st.max())} "
                                   "(2 = zero theta, 4 = tape/bond mismatch)")
        b.check_status()
        return grads


# -- rotation gates -------------------------------------------------------------------
def rot_gates(angles: torch.Tensor) -> torch.Tensor:
    """RZ(phi) RY(theta) with RY = exp(-i theta Y/2), RZ = exp(-i phi Z/2); angles (..., 2) -> (..., 2, 2)."""
    th, ph = angles[..., 0], angles[..., 1]
    c, s = torch.cos(0.5 * th), torch.sin(0.5 * th)
    em, ep = torch.exp(-0.5j * ph), torch.exp(0.5j * ph)
    row0 = torch.stack([em * c, -em * s], -1)
    row1 = torch.stack([ep * s, ep * c], -1)
    return torch.stack([row0, row1], -2)


def rot_angle_grads(angles: torch.Tensor, gbar: torch.Tensor) -> torch.Tensor:
    """dL/d(theta, phi) = Re sum conj(G_bar) dG/d(theta, phi) for G = rot_gates(angles)."""
    th, ph = angles[..., 0], angles[..., 1]
    c, s = torch.cos(0.5 * th), torch.sin(0.5 * th)
    em, ep = torch.exp(-0.5j * ph), torch.exp(0.5j * ph)
    dth = torch.stack([torch.stack([-0.5 * em * s, -0.5 * em * c], -1),
                       torch.stack([0.5 * ep * c, -0.5 * ep * s], -1)], -2)
    g = rot_gates(angles)
    sign = torch.tensor([[-0.5j], [0.5j]], dtype=torch.complex128, device=angles.device)
    dph = g * sign
    gt = torch.real(torch.sum(torch.conj(gbar) * dth, dim=(-2, -1)))
    gp = torch.real(torch.sum(torch.conj(gbar) * dph, dim=(-2, -1)))
    return torch.stack([gt, gp], -1)


def _pairs_layer(batch: MPSBatch, nvec: int, n: int, start: int, gate: np.ndarray) -> PairBatch:
    left = np.arange(start, n - 1, 2, dtype=np.int32)
    ci = np.repeat(np.arange(nvec, dtype=np.int32), len(left))
    si = np.tile(left, nvec)
    return batch.make_pairs(ci, si, np.repeat(gate[None], len(si), 0))


class HEAEnergy:
    """Hardware-efficient ansatz energies and their adjoint gradient.

    ``nvec`` parameter vectors of shape (layers, n, 2) -- [..., 0] the RY
    angle, [..., 1] the RZ angle of every site -- run as ``nvec`` independent
    chains of one batch; each ansatz layer is RY, RZ on every site (one
    fused gate RZ RY), then CZ on the even pairs, then CZ on the odd pairs.
    Loss per vector: the transverse-field Ising energy
    -J sum Z_i Z_{i+1} - h sum X_i, normalised by <psi|psi>.
    """

    def __init__(self, n: int, layers: int, nvec: int, chi_max: int = 32, cutoff: float = 1e-12,
                 precision: str = "fp64", J: float = 1.0, h: float = 1.0,
                 device: Union[str, torch.device] = "cuda", checkpoint: Union[bool, str] = "auto"):
        self.n, self.layers, self.nvec = int(n), int(layers), int(nvec)
        self.batch = MPSBatch([n] * nvec, chi_max, cutoff, precision=precision, device=device)
        self.device = self.batch.device
        self.engine = AdjointEngine(self.batch, tfim_mpo(n, J, h), checkpoint=checkpoint)
        ci = np.repeat(np.arange(nvec, dtype=np.int32), n)
        si = np.tile(np.arange(n, dtype=np.int32), nvec)
        ops = np.stack([ci, si, np.arange(nvec * n, dtype=np.int32), np.zeros(nvec * n, np.int32)], 1)
        self.ops = torch.from_numpy(np.ascontiguousarray(ops)).to(self.device)
        self.even = _pairs_layer(self.batch, nvec, n, 0, _CZ)
        self.odd = _pairs_layer(self.batch, nvec, n, 1, _CZ)
        self.gates = torch.zeros(layers, nvec * n, 2, 2, dtype=torch.complex128, device=self.device)
        cap = self.batch.chi_cap
        self.groups = [[Step1Q(self.ops, self.gates[l], f"rot{l}"), Step2Q(self.even, cap), Step2Q(self.odd, cap)]
                       for l in range(layers)]

    def _reset(self) -> None:
        b = self.batch
        b.sites.zero_()
        b.sites[:, 0] = 1.0
        b.bonds.fill_(1)
        b.norm_logs.zero_()
        b.status_acc.zero_()

    def _set_angles(self, angles) -> torch.Tensor:
        a = torch.as_tensor(angles, dtype=torch.float64, device=self.device)
        if a.shape != (self.nvec, self.layers, self.n, 2):
            raise ValueError(f"angles must have shape {(self.nvec, self.layers, self.n, 2)}, got {tuple(a.shape)}")
        self.gates.copy_(rot_gates(a.permute(1, 0, 2, 3).reshape(self.layers, self.nvec * self.n, 2)))
        return a

    def forward(self, angles) -> torch.Tensor:
        """Energies (nvec,) with checkpoints kept for a following backward()."""
        self._set_angles(angles)
        self._reset()
        self.engine.forward(self.groups)
        return self.engine.energy().clone()

    def backward(self, angles, weights: Optional[torch.Tensor] = None) -> torch.Tensor:
        """sum_c weights[c] dL_c/dangles_c, shape (nvec, layers, n, 2), for the last forward()."""
        a = torch.as_tensor(angles, dtype=torch.float64, device=self.device)
        grads = self.engine.backward(weights)
        out = torch.empty(self.layers, self.nvec * self.n, 2, dtype=torch.float64, device=self.device)
        flat = a.permute(1, 0, 2, 3).reshape(self.layers, self.nvec * self.n, 2)
        for l in range(self.layers):
            out[l] = rot_angle_grads(flat[l], grads[f"rot{l}"])
        return out.reshape(self.layers, self.nvec, self.n, 2).permute(1, 0, 2, 3).contiguous()

    def energy_and_grad(self, angles, weights: Optional[torch.Tensor] = None):
        e = self.forward(angles)
        return e, self.backward(angles, weights)


class HEAEnergyFunction(torch.autograd.Function):
    """torch.autograd.Function over HEAEnergy: angles (nvec, layers, n, 2) -> energies (nvec,).

    The forward keeps per-layer checkpoints; the backward recomputes every
    layer with tapes and runs the hand-written adjoint (no torch autograd
    graph through the state)."""

    @staticmethod
    def forward(ctx, angles: torch.Tensor, model: HEAEnergy) -> torch.Tensor:
        ctx.model = model
        ctx.save_for_backward(angles)
        return model.forward(angles.detach())

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (angles,) = ctx.saved_tensors
        g = ctx.model.backward(angles.detach(), grad_out.detach())
        return g.to(angles.device), None


class XXZInitialStateGradient:
    """d/d(initial Bloch angles) of sum_i <Z_i Z_{i+1}> after a Trotterised XXZ evolution.

    Initial state: site k = cos(theta_k/2)|0> + e^{i phi_k} sin(theta_k/2)|1>;
    then ``steps`` second-order Trotter steps (half step on odd bonds, full
    step on even bonds, half step on odd bonds) of H = Jxy (XX + YY) + Jz ZZ
    with exact exp(-i dt h) bond gates; checkpoints per Trotter step.
    """

    def __init__(self, n: int, steps: int, dt: float = 0.05, jxy: float = 1.0, jz: float = 0.5,
                 chi_max: int = 64, cutoff: float = 1e-10, precision: str = "fp64",
                 device: Union[str, torch.device] = "cuda", checkpoint: Union[bool, str] = "auto"):
        self.n, self.steps = int(n), int(steps)
        self.batch = MPSBatch([n], chi_max, cutoff, precision=precision, device=device)
        self.device = self.batch.device
        self.engine = AdjointEngine(self.batch, zz_mpo(n), checkpoint=checkpoint)
        layers = xxz_trotter_layers(n, steps, dt, jxy, jz)
        cap = self.batch.chi_cap
        pbs = [self.batch.make_pairs(np.zeros(len(L.sites), np.int32), L.sites, L.gates) for L in layers]
        self.groups = [[Step2Q(pbs[3 * t + j], cap) for j in range(3)] for t in range(steps)]

    def _set_state(self, angles: torch.Tensor) -> None:
        b = self.batch
        th, ph = angles[:, 0], angles[:, 1]
        b.sites.zero_()
        b.sites[:, 0] = torch.cos(0.5 * th).to(torch.complex128)
        b.sites[:, 1] = torch.exp(1j * ph) * torch.sin(0.5 * th)
        b.bonds.fill_(1)
        b.norm_logs.zero_()
        b.status_acc.zero_()

    def energy(self, angles) -> float:
        a = torch.as_tensor(angles, dtype=torch.float64, device=self.device)
        self._set_state(a)
        for g in self.groups:
            for st in g:
                self.engine._run(st)
        return float(self.engine.energy().item())

    def energy_and_grad(self, angles) -> Tuple[float, torch.Tensor]:
        a = torch.as_tensor(angles, dtype=torch.float64, device=self.device)
        if a.shape != (self.n, 2):
            raise ValueError(f"angles must have shape ({self.n}, 2)")
        self._set_state(a)
        self.engine.forward(self.groups)
        self.engine.backward()
        e = float(self.engine.loss.item())
        c0 = self.engine.cot[:, 0]
        c1 = self.engine.cot[:, 1]
        th, ph = a[:, 0], a[:, 1]
        eph = torch.exp(1j * ph)
        d0_th = -0.5 * torch.sin(0.5 * th)
        d1_th = 0.5 * eph * torch.cos(0.5 * th)
        d1_ph = 1j * eph * torch.sin(0.5 * th)
        g_th = torch.real(torch.conj(c0) * d0_th + torch.conj(c1) * d1_th)
        g_ph = torch.real(torch.conj(c1) * d1_ph)
        return e, torch.stack([g_th, g_ph], 1)
