"""Error types of the Debye path.

Mirrors the reference's ``crate::Error`` variants that the Debye path can
raise (src/error.rs:16-74) and the Python exception classes its pyo3 binding
maps them to (pripps-py/src/lib.rs:805-818): ``QOutOfRange``, ``Validation``,
``Usage`` and ``UndefinedFormFactor`` surface as ``ValueError``; ``Internal``
as ``RuntimeError``. Device-side failures of the CUDA backend (a bounded wait
that expired, an allocation refused by the memory budget) have no reference
counterpart and surface as ``DeviceError`` (a ``RuntimeError``).
"""


class PrippsError(Exception):
    """Base class of every error raised by this package."""


class QOutOfRange(PrippsError, ValueError):
    """A form factor was evaluated outside its inclusive q range
    (src/formfactor.rs:188-193)."""

    def __init__(self, q, lo, hi):
        super().__init__(f"q = {q} is outside the form factor's range [{lo}, {hi}]")
        self.q, self.lo, self.hi = q, lo, hi


class ValidationError(PrippsError, ValueError):
    """Invalid input data (Error::Validation)."""


class UsageError(PrippsError, ValueError):
    """Invalid combination of options (Error::Usage)."""


class UndefinedFormFactor(PrippsError, ValueError):
    """A symbolic form factor names an undefined species
    (Error::UndefinedFormFactor)."""


class InternalError(PrippsError, RuntimeError):
    """Broken internal invariant (Error::Internal)."""


class DeviceError(PrippsError, RuntimeError):
    """The CUDA backend reported a failure (error code and message from
    ``pd_last_error``)."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code
