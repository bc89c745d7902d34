"""Exception types matching the Julia exceptions thrown on the IMEX path.

The C-ABI returns status codes; ``raise_status`` turns them into these classes so
that host code sees the same failure kinds as the reference:

====================  =====================  ==========================================
status                Python class           Julia exception (example site)
====================  =====================  ==========================================
EFSI_ARG              ArgumentError          ArgumentError (TimeIntegrationIMEX.jl:1121)
EFSI_DIM              DimensionMismatch      DimensionMismatch (TimeIntegrationIMEX.jl:500)
EFSI_SOLVE            SolverError            ErrorException (Projection.jl:281, :293)
EFSI_DOMAIN           DomainError            DomainError (StructureTensor.jl:491)
EFSI_CUDA             CUDAError              (device failure; no Julia counterpart)
EFSI_UNSUPPORTED      UnsupportedError       (valid input outside the device step)
====================  =====================  ==========================================
"""


class EFSIError(Exception):
    """Base class of every error raised through the C-ABI."""


class ArgumentError(EFSIError, ValueError):
    pass


class DimensionMismatch(EFSIError, ValueError):
    pass


class SolverError(EFSIError, RuntimeError):
    pass


class DomainError(EFSIError, ValueError):
    pass


class CUDAError(EFSIError, RuntimeError):
    pass


class UnsupportedError(EFSIError, NotImplementedError):
    pass


_BY_CODE = {1: ArgumentError, 2: DimensionMismatch, 3: SolverError, 4: DomainError, 5: CUDAError,
            6: UnsupportedError}


def raise_status(code: int, message: str) -> None:
    if code == 0:
        return
    raise _BY_CODE.get(code, EFSIError)(message or f"status {code}")
