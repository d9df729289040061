"""jaqsi_b200 — a B200 (sm_100a) execution backend for jaqsi's circuit path.

Drop-in surface of the reference's simulation layer: record a circuit with the
gate classes below inside ``Script(f, n_qubits)`` and call
``.execute(type="expval"|"probs"|"state"|"density", obs=..., args=...)``.
Execution runs in libjqsim.so (hand-written CUDA for sm_100a) through a
ctypes C ABI; torch tensors are used only at the boundary.
"""
from jaqsi_b200.operations import GateStructure, Hermitian, Operation, cdtype, set_default_dtype
from jaqsi_b200.gateset import (
    CCX, CRX, CRY, CRZ, CSWAP, CX, CY, CZ, H, RX, RXX, RY, RYY, RZ, RZX, RZZ, S, SWAP, Barrier,
    ControlledPauliRot, ControlledPhaseShift, DiagonalQubitUnitary, Id, PauliRot, PauliX, PauliY, PauliZ,
    RandomUnitary, Rot, build_parity_observable,
)
from jaqsi_b200.noise import (
    AmplitudeDamping, BitFlip, DepolarizingChannel, KrausChannel, PhaseDamping, PhaseFlip, QubitChannel,
    ThermalRelaxationError,
)
from jaqsi_b200.script import Script, make_hashable
from jaqsi_b200.tape import copy_to_tape, recording, shift_and_append
from jaqsi_b200 import simulation
from jaqsi_b200.batch import BatchedGradients
from jaqsi_b200.evolution import Evolution, ParametrizedHamiltonian, PendingEvolution, resolve_pending

__version__ = "0.1.0"

__all__ = [
    "Script", "Operation", "Hermitian", "GateStructure", "cdtype", "set_default_dtype", "make_hashable",
    "recording", "copy_to_tape", "shift_and_append", "simulation", "build_parity_observable", "BatchedGradients",
    "Id", "PauliX", "PauliY", "PauliZ", "H", "S", "SWAP", "RX", "RY", "RZ", "Rot", "CX", "CY", "CZ", "CCX",
    "CSWAP", "CRX", "CRY", "CRZ", "ControlledPhaseShift", "PauliRot", "RXX", "RYY", "RZZ", "RZX",
    "ControlledPauliRot", "DiagonalQubitUnitary", "RandomUnitary", "Barrier",
    "KrausChannel", "BitFlip", "PhaseFlip", "DepolarizingChannel", "AmplitudeDamping", "PhaseDamping",
    "ThermalRelaxationError", "QubitChannel",
    "Evolution", "ParametrizedHamiltonian", "PendingEvolution", "resolve_pending",
]
