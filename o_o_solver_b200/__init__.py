"""B200 implementation of O_o_Solver's numeric hot path: the supernodal multifrontal LDL^T factorisation and its
solves on the GPU, behind the reference's factorisation interface (SymbolicFactor, SupernodalFactor.factorise,
FactorSolve.solve), the shifted pencils of its eigenvalue analyses (SparsePencil, BucklingPencil) and a C ABI
(include/oos_gpu.h)."""

from .linalg import (  # noqa: F401
    BucklingPencil,
    FactorOptions,
    FactorSolve,
    Inertia,
    MemoryBudgetError,
    PartialFactor,
    PivotPolicy,
    ShiftFactorisation,
    SingularityError,
    SolverError,
    SparsePencil,
    SupernodalFactor,
    SymbolicFactor,
    SymmetricCsc,
    device_count,
)
