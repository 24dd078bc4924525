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


class ValueLayout(enum.IntEnum):
    """Order of the 9 * nnzb values of a 3x3 block CSR matrix."""

    RowStrips = capi.SDX_BSR_ROW_STRIPS  # BlockSparseMatrix<T,3>::Values() (block_sparse_matrix.h:459-475)
    Blocks = capi.SDX_BSR_BLOCKS         # 9 contiguous row-major values per block (cuSPARSE BSR)


@dataclasses.dataclass
class BlockSparseMatrix:
    """3x3 block CSR, as the reference's BlockSparseMatrix<T,3> (block_sparse_matrix.h:63): Pointers(),
    Indices() and Values(). By default the values are in the reference's own row-strip layout: block row br
    with nb blocks is one row-major 3 x 3nb strip at 9 row_ptr[br], entry (lr, lc) of its k-th block at
    3 (lr nb + k) + lc. `layout=ValueLayout.Blocks` takes contiguous 3x3 blocks instead."""

    row_ptr: np.ndarray  # int64 (or int32), block_rows + 1
    col: np.ndarray      # int32, nnzb
    values: np.ndarray   # 9 * nnzb float32 or float64 (any shape) in `layout`
    layout: ValueLayout = ValueLayout.RowStrips

    @property
    def block_rows(self) -> int:
        return int(self.row_ptr.size - 1)

    @staticmethod
    def from_blocks(row_ptr, col, blocks, layout: ValueLayout = ValueLayout.RowStrips) -> "BlockSparseMatrix":
        """Matrix from (nnzb, 3, 3) blocks, its values stored in `layout`."""
        blocks = np.asarray(blocks).reshape(-1, 3, 3)
        if layout == ValueLayout.Blocks:
            return BlockSparseMatrix(np.asarray(row_ptr), np.asarray(col), blocks.reshape(-1).copy(), layout)
        return BlockSparseMatrix(np.asarray(row_ptr), np.asarray(col), blocks_to_strips(row_ptr, blocks), layout)


def blocks_to_strips(row_ptr, blocks) -> np.ndarray:
    """Values of (nnzb, 3, 3) blocks in the reference's row-strip order."""
    row_ptr = np.asarray(row_ptr, np.int64)
    blocks = np.asarray(blocks).reshape(-1, 3, 3)
    out = np.empty(9 * blocks.shape[0], blocks.dtype)
    for br in range(row_ptr.size - 1):
        b0, b1 = int(row_ptr[br]), int(row_ptr[br + 1])
        # strip[lr, 3k + lc] = block k [lr, lc]
        out[9 * b0:9 * b1] = blocks[b0:b1].transpose(1, 0, 2).reshape(-1)
    return out


def strips_to_blocks(row_ptr, values) -> np.ndarray:
    """(nnzb, 3, 3) blocks of values in the reference's row-strip order."""
    row_ptr = np.asarray(row_ptr, np.int64)
    values = np.asarray(values).reshape(-1)
    nnzb = int(row_ptr[-1])
    out = np.empty((nnzb, 3, 3), values.dtype)
    for br in range(row_ptr.size - 1):
        b0, b1 = int(row_ptr[br]), int(row_ptr[br + 1])
        out[b0:b1] = values[9 * b0:9 * b1].reshape(3, b1 - b0, 3).transpose(1, 0, 2)
    return out


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
        prm.value_layout = int(A.layout)
        rc = capi.lib().sdx_pcg_solve_ctx(self._ctx, n, col.size, capi.ptr(row_ptr, capi._lp),
                                          capi.ptr(col, capi._ip), vals.ctypes.data_as(C.c_void_p), vt,
                                          capi.ptr(b), capi.ptr(x), int(hint), C.byref(prm), C.byref(st))
        if rc == -1:
            raise ValueError(capi.lib().sdx_last_error().decode())
        capi.check(rc)
        return LinearSolverStatus(st.num_iter, st.residual_norm, st.relative_residual_norm,
                                  LinearSolverConvergenceStatus(st.convergence))
