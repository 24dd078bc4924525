"""LinearSolver mirror: the reference's linear-solver boundary on the GPU.

Mirrors mochi::LinearSolver<T>::Solve (mochi_core/include/mochi_core/solvers/linear_solver.h:321-496)
for solverType = CudaCG with the Jacobi / block-Jacobi preconditioner and the residual-L2 stop test:
same parameter names and meaning (KrylovSolverParams, krylov_solver.h:43-82), same status struct
(LinearSolverStatus, krylov_solver.h:85-116), and convergence reported through the status rather than
by exceptions. Invalid arguments raise ValueError (the reference asserts).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum

import numpy as np

from . import capi


class InitialGuessHint(enum.IntEnum):
    Unknown = capi.SDX_GUESS_UNKNOWN
    Zero = capi.SDX_GUESS_ZERO


class PreconditionerType(enum.IntEnum):
    None_ = capi.SDX_PREC_NONE
    Jacobi = capi.SDX_PREC_JACOBI
    BlockJacobi = capi.SDX_PREC_BLOCK_JACOBI


class LinearSolverConvergenceStatus(enum.IntEnum):
    None_ = 0
    Converged = 1
    Stopped = 2
    Diverged = 3


@dataclasses.dataclass
class KrylovSolverParams:
    """Defaults as KrylovSolverParams / LinearSolverParams (linear_solver_params.h:344-418)."""

    relTol: float = 1e-5
    absTol: float = 1e-9
    relDivTol: float = 1e10
    maxIter: int = 500
    preconditionerType: PreconditionerType = PreconditionerType.Jacobi
    abortIfNotSpd: bool = False
    usePolakRibiere: bool = True
    replaceEvery: int = 32  # FP64 true-residual replacement period (B200 mixed-precision CG)

    def to_c(self) -> capi.LinearParams:
        p = capi.LinearParams()
        p.rel_tol, p.abs_tol, p.rel_div_tol = self.relTol, self.absTol, self.relDivTol
        p.max_iter = int(self.maxIter)
        p.preconditioner = int(self.preconditionerType)
        p.abort_if_not_spd = int(self.abortIfNotSpd)
        p.polak_ribiere = int(self.usePolakRibiere)
        p.replace_every = int(self.replaceEvery)
        return p


@dataclasses.dataclass
class LinearSolverStatus:
    numIterDone: int
    residualNorm: float
    relativeResidualNorm: float
    convergence: LinearSolverConvergenceStatus


@dataclasses.dataclass
class BlockSparseMatrix:
    """3x3 block CSR (block-contiguous row-major blocks)."""

    row_ptr: np.ndarray  # int64, block_rows + 1
    col: np.ndarray      # int32, nnzb
    values: np.ndarray   # (nnzb, 3, 3) float32 or float64

    @property
    def block_rows(self) -> int:
        return int(self.row_ptr.size - 1)


class LinearSolver:
    """GPU Jacobi-PCG behind the reference's LinearSolver::Solve signature."""

    def __init__(self, params: KrylovSolverParams | None = None, device: int = 0):
        self.params = params or KrylovSolverParams()
        L = capi.lib()
        self._ctx = L.sdx_create(device)
        if not self._ctx:
            raise capi.SdxError(L.sdx_last_error().decode())

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx:
            capi.lib().sdx_destroy(ctx)
            self._ctx = None

    def GetParams(self) -> KrylovSolverParams:
        return self.params

    def SetParams(self, params: KrylovSolverParams):
        self.params = params

    def Solve(self, A: BlockSparseMatrix, b: np.ndarray, x: np.ndarray, hasOperatorChanged: bool = True,
              hint: InitialGuessHint = InitialGuessHint.Unknown) -> LinearSolverStatus:
        """Solve A x = b. x (float64, 3 * block_rows) is the initial guess and receives the solution."""
        n = A.block_rows
        row_ptr = np.ascontiguousarray(A.row_ptr, np.int64)
        col = np.ascontiguousarray(A.col, np.int32)
        vals = np.ascontiguousarray(A.values)
        if vals.dtype == np.float32:
            vt = capi.SDX_F32
        elif vals.dtype == np.float64:
            vt = capi.SDX_F64
        else:
            raise ValueError("values must be float32 or float64")
        if vals.size != 9 * col.size:
            raise ValueError("values must hold 9 entries per block")
        b = np.ascontiguousarray(b, np.float64).reshape(-1)
        if b.size != 3 * n or x.size != 3 * n or x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("b and x must be float64 vectors of length 3 * block_rows")
        st = capi.LinearStatus()
        prm = self.params.to_c()
        rc = capi.lib().sdx_pcg_solve_ctx(self._ctx, n, col.size, capi.ptr(row_ptr, capi._lp),
                                          capi.ptr(col, capi._ip), vals.ctypes.data_as(C.c_void_p), vt,
                                          capi.ptr(b), capi.ptr(x), int(hint), C.byref(prm), C.byref(st))
        if rc == -1:
            raise ValueError(capi.lib().sdx_last_error().decode())
        capi.check(rc)
        return LinearSolverStatus(st.num_iter, st.residual_norm, st.relative_residual_norm,
                                  LinearSolverConvergenceStatus(st.convergence))
