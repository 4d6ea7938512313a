"""B200 (sm_100a) MPS two-site update: CUDA kernels behind a C ABI, host API mirroring mps_core.MPSState."""
from .gates import (GATE_MATRICES, SINGLE_QUBIT_GATES, TWO_QUBIT_GATES, gate_1q, gate_2q, permute_2q,
                    swap_route)

__all__ = ["GATE_MATRICES", "SINGLE_QUBIT_GATES", "TWO_QUBIT_GATES", "gate_1q", "gate_2q", "permute_2q",
           "swap_route", "MPSState", "MPSBatch", "MPSSimulator", "MPSResult", "Circuit", "HEAEnergy",
           "HEAEnergyFunction"]


def __getattr__(name):
    # torch and the CUDA library are only needed for the device classes
    if name in ("MPSState", "MPSBatch", "PairBatch", "FlowBatch", "ThetaBatch"):
        from . import mps
        return getattr(mps, name)
    if name in ("MPSSimulator", "MPSResult", "Circuit"):
        from . import compiler
        return getattr(compiler, name)
    if name in ("HEAEnergy", "HEAEnergyFunction", "XXZInitialStateGradient"):
        from . import adjoint
        return getattr(adjoint, name)
    raise AttributeError(name)
