"""pylcm_b200: a B200-native backward-induction solver with PyLCM's model API.

Declare a model with the same objects as PyLCM (``Model``, ``Regime``, grids,
processes, ``MarkovTransition``, ``categorical``) and call
``model.solve(params=...)`` / ``model.simulate(...)``.  Model functions are
lowered to CUDA C, compiled with NVRTC for sm_100a and run by the kernels in
``pylcm_b200/csrc`` through the C-ABI library ``liblcmx.so``.
"""

from pylcm_b200 import jnp
from pylcm_b200.ages import AgeGrid
from pylcm_b200.exceptions import (
    AdmissionError,
    GridInitializationError,
    InvalidInitialConditionsError,
    InvalidParamsError,
    InvalidRegimeTransitionProbabilitiesError,
    InvalidStateTransitionProbabilitiesError,
    InvalidValueFunctionError,
    KernelError,
    ModelInitializationError,
    PyLCMError,
    RegimeInitializationError,
    TracingError,
)
from pylcm_b200.grids import (
    DiscreteGrid,
    IrregSpacedGrid,
    LinSpacedGrid,
    LogSpacedGrid,
    PiecewiseGridSegment,
    PiecewiseLinSpacedGrid,
    PiecewiseLogSpacedGrid,
    categorical,
)
from pylcm_b200.model import Model
from pylcm_b200.processes import (
    LogNormalIIDProcess,
    NormalIIDProcess,
    NormalMixtureIIDProcess,
    RouwenhorstAR1Process,
    TauchenAR1Process,
    TauchenNormalMixtureAR1Process,
    UniformIIDProcess,
)
from pylcm_b200.regime import (
    ConsumptionSavingsRegime,
    ExtremeValueTasteShocks,
    LiquidMargin,
    MarkovTransition,
    Regime,
)
from pylcm_b200.solvers import (
    DCEGM,
    EGM,
    NEGM,
    ExactEnvelope,
    FUESEnvelope,
    GridSearch,
    LTMEnvelope,
    MSSEnvelope,
    RFCEnvelope,
)

__all__ = [
    "DCEGM",
    "EGM",
    "NEGM",
    "AdmissionError",
    "AgeGrid",
    "ConsumptionSavingsRegime",
    "DiscreteGrid",
    "ExtremeValueTasteShocks",
    "ExactEnvelope",
    "FUESEnvelope",
    "LTMEnvelope",
    "MSSEnvelope",
    "RFCEnvelope",
    "GridInitializationError",
    "GridSearch",
    "InvalidInitialConditionsError",
    "InvalidParamsError",
    "InvalidRegimeTransitionProbabilitiesError",
    "InvalidStateTransitionProbabilitiesError",
    "InvalidValueFunctionError",
    "IrregSpacedGrid",
    "KernelError",
    "LinSpacedGrid",
    "LiquidMargin",
    "LogNormalIIDProcess",
    "LogSpacedGrid",
    "PiecewiseGridSegment",
    "PiecewiseLinSpacedGrid",
    "PiecewiseLogSpacedGrid",
    "MarkovTransition",
    "Model",
    "ModelInitializationError",
    "NormalIIDProcess",
    "NormalMixtureIIDProcess",
    "PyLCMError",
    "Regime",
    "RegimeInitializationError",
    "RouwenhorstAR1Process",
    "TauchenAR1Process",
    "TauchenNormalMixtureAR1Process",
    "TracingError",
    "UniformIIDProcess",
    "categorical",
    "jnp",
]
