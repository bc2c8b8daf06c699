"""Exception classes, named after the reference's (``src/lcm/exceptions.py``)."""


class PyLCMError(Exception):
    """Base class for all errors raised by this package."""


class GridInitializationError(PyLCMError):
    """A grid or process was declared with invalid arguments."""


class ModelInitializationError(PyLCMError):
    """A model could not be built from its regimes."""


class RegimeInitializationError(ModelInitializationError):
    """A regime was declared with invalid arguments."""


class InvalidParamsError(PyLCMError):
    """The params passed to solve/simulate do not match the model."""


class InvalidRegimeTransitionProbabilitiesError(PyLCMError):
    """Regime transition probabilities are non-finite, outside [0, 1], do not
    sum to one, or reach a regime that is inactive next period."""


class InvalidStateTransitionProbabilitiesError(PyLCMError):
    """A stochastic state transition returned an invalid probability row."""


class InvalidValueFunctionError(PyLCMError):
    """A solved value function contains NaN."""


class InvalidInitialConditionsError(PyLCMError):
    """The initial conditions passed to simulate do not match the model."""


class TracingError(PyLCMError):
    """A model function uses a construct the CUDA lowering does not support."""


class KernelError(PyLCMError):
    """The native library reported a failure (compile, launch, bounded wait, ...)."""

    def __init__(self, status: int, message: str) -> None:
        super().__init__(f"[lcmx status {status}] {message}")
        self.status = status


class AdmissionError(PyLCMError, MemoryError):
    """A serving request does not fit the configured HBM budget (no
    counterpart in the reference, which has no serving layer)."""
