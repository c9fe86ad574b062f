"""Foundation records of the host API: the health error, the fallback reasons, Neumaier totals.

Mirrors src/Foundation/Foundation.jl: `NumericalHealthError` (:21-36), `effective_eps` (:44-45), `CompensatedSum` /
`total` (:48-68) and `FALLBACK_REASONS` (:71-75).
"""
from __future__ import annotations

import numpy as np

EPS = float(np.finfo(np.float64).eps)  # effective_eps(Float64)

# src/Foundation/Foundation.jl:71-75, in the reference's order (index 1-based there).
FALLBACK_REASONS = [
    "CUDA.jl not loadable", "no functional device", "kernel does not compile for the element type",
    "device out of memory", "NumericalHealthError raised only on the GPU", "reducer is CPU-only",
    "GPU not faster for the element type", "launch exceeds the display watchdog", "device lost",
]


class NumericalHealthError(Exception):
    """A numerical health check failed (Foundation.jl:21-36): `what` is the kind ("state", "deviation matrix",
    "orthogonality", "orthonormalisation breakdown", ...), `value` / `threshold` the offending value and its bound,
    `step` the global step, `orbit` the 1-based orbit id, `backend` "cpu" or "gpu", `column` the deviation column
    (0 when none)."""

    def __init__(self, what: str, value: float, threshold: float, step: int, orbit: int, backend: str,
                 column: int = 0):
        self.what, self.value, self.threshold = what, float(value), float(threshold)
        self.step, self.orbit, self.backend, self.column = int(step), int(orbit), backend, int(column)
        super().__init__(str(self))

    def __str__(self) -> str:  # Base.showerror, Foundation.jl:33-36
        return (f"NumericalHealthError: {self.what} = {self.value} (threshold {self.threshold}) at step "
                f"{self.step}, orbit {self.orbit}, backend {self.backend}")

    def __eq__(self, other) -> bool:
        if not isinstance(other, NumericalHealthError):
            return NotImplemented
        same = lambda a, b: (a == b) or (np.isnan(a) and np.isnan(b))  # noqa: E731
        return (self.what == other.what and same(self.value, other.value) and same(self.threshold, other.threshold)
                and self.step == other.step and self.orbit == other.orbit and self.backend == other.backend
                and self.column == other.column)

    __hash__ = None


def total(s: float, c: float) -> float:
    """`total(CompensatedSum)` = s + c (Foundation.jl:68), in binary64."""
    return float(np.float64(s) + np.float64(c))


class DimensionMismatch(ValueError):
    """Julia's `DimensionMismatch`: two arrays of different sizes met in an elementwise operation (StaticArrays
    throws it for `SVector{m} + SVector{n}`, m != n)."""


class DeviceError(RuntimeError):
    """A device call failed; `reason` is the 1-based FALLBACK_REASONS index it maps to (3, 4 or 9), as
    `_fallback_reason` classifies device exceptions (src/Tangent/propagate.jl:121-129)."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.reason = {-2: 2, -3: 3, -4: 4, -8: 8, -9: 9}.get(code, 0)
        super().__init__(f"libchaoslab_b200 error {code}: {message}")
