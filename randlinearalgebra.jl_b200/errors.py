"""Exceptions named after the Julia exceptions the reference throws.

The messages are the reference's own (constructor checks, src/helpers/mul_dim_checks.jl,
src/Compressors.jl:146-153 and :314).
"""


class RLAError(RuntimeError):
    """A library failure with no Julia counterpart (CUDA error, out of memory, ...)."""


class ArgumentError(ValueError):
    """Julia's ArgumentError."""


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch."""


class DomainError(ValueError):
    """Julia's DomainError."""
