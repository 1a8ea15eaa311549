"""mossquantum_b200: a B200 (sm_100a) dense FP64 simulation backend for MOSSQuantum.

Host-side mirror of MOSSQuantum's backend, state, circuit, observable and gradient APIs,
driving hand-written CUDA kernels through the C ABI in include/mossb200.h.
"""
from ._native import BackendError, BudgetExceeded, UnsupportedOperation, init, launch_count, memory_info, synchronize
from .backend import (B200Backend, SimulationResult, apply, apply_, apply_observable, backend, counts, expectation,
                      probabilities, sample, simulate, supports)
from .channels import (AmplitudeDamping, BitFlip, BitPhaseFlip, Depolarizing, GeneralizedAmplitudeDamping, MixedUnitary,
                       PauliChannel, PhaseDamping, PhaseFlip, QuantumMap, ResetChannel, ThermalRelaxation)
from .circuit import ParameterMap, QCircuit, accumulate_parameter_gradients, bind_parameters
from .gates import (CCPHASEGate, CNOTGate, CONTROLCONTROLGate, CONTROLGate, CPHASEGate, CRxGate, CRyGate, CRzGate,
                    CZGate, FREDKINGate, FSIMGate, HGate, PHASEGate, QuantumGate, RxGate, RyGate, RzGate, SGate,
                    SWAPGate, TGate, TOFFOLIGate, XGate, YGate, ZGate, AdjointQuantumGate, gate, iSWAPGate,
                    sqrtXGate, sqrtYGate, U3)
from .objectives import (AdjointGradient, B200AdjointGradient, BatchExpectationObjective, ExpectationObjective,
                         UnsupportedGradient, differentiable_value, evaluate, evaluate_batch, supports_gradient,
                         value_and_gradient, value_and_pullback)
from .fusion import fuse_gates
from .measurement import (MeasurementRecord, QMeasure, QSelect, discrete_sample, measure, measure_, post_select,
                          post_select_)
from .operators import QubitsOperator, QubitsTerm
from .reduced import fidelity, inner, partial_tr, trace
from .sampled import (FiniteDifference, GradientEstimate, ParameterShift, SPSAGradient, estimate_gradient,
                      parameter_shift_rule)
from .trajectories import CountsResult, DensityMatrixEvolution, KrausTrajectory, execute, run_trajectories
from .states import (BatchDensityMatrix, BatchStateVector, DensityMatrix, HostConversionError, StateVector)

__all__ = [k for k in dir() if not k.startswith("_")]
