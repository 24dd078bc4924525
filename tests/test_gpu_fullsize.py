"""Full-size checks on the measured workload (the 64^3 body with 5 capsules), through properties that do
not need the oracle to run at full size: the Newton residual reaches rel 1e-6, the assembled Hessian is
symmetric, the linear solve meets rel 1e-6 on the FP64 true residual of the FP32 matrix, and the
contact pairs are bit-identical to the oracle's detection at the same state."""
import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg1_world():
    from project_superdex_b200.soft_body import SoftBodyWorld
    bodies, cfg = scenes.config1()
    w = SoftBodyWorld(bodies, cfg, newton_abs_tol=1e-9)
    w.step(2)
    yield w, bodies[0], cfg
    w.close()


def test_newton_converges_to_rel_1e6(cfg1_world):
    w, b, cfg = cfg1_world
    st = w.stats()[0]
    assert st["convergence"] == 1
    assert st["res_norm"] <= 1e-6 * st["res_norm0"]
    assert st["n_contacts"] > 0


def test_hessian_symmetric_and_linear_solve_true_residual(cfg1_world):
    import scipy.sparse as sp
    from project_superdex_b200.linear_solver import (BlockSparseMatrix, InitialGuessHint, KrylovSolverParams,
                                                     LinearSolver, ValueLayout)
    w, b, cfg = cfg1_world
    u, v, t = w.get_state()
    a = w.assemble(None, t=t + cfg.dt)
    rp, col = w.pattern()
    H = a["H"].astype(np.float64)
    n = b.n_nodes
    # block CSR -> scalar CSR
    rows = np.repeat(np.arange(n), np.diff(rp))
    r3 = (3 * rows[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
    c3 = (3 * col[:, None, None].astype(np.int64) + np.arange(3)[None, None, :]).repeat(3, axis=1)
    A = sp.csr_matrix((H.reshape(-1), (r3.reshape(-1), c3.reshape(-1))), shape=(3 * n, 3 * n))
    asym = abs(A - A.T).max()
    assert asym <= 1e-5 * abs(A).max()
    g = a["g"]
    x = np.zeros_like(g)
    st = LinearSolver(KrylovSolverParams(relTol=1e-6, maxIter=20000)).Solve(BlockSparseMatrix(rp, col, a["H"], ValueLayout.Blocks), g, x,
                                                                            hint=InitialGuessHint.Zero)
    assert st.convergence == 1
    true_rel = np.linalg.norm(g - A @ x) / np.linalg.norm(g)
    assert true_rel <= 1.01e-6


def test_contact_pairs_bit_exact_at_full_size(cfg1_world, oracle):
    w, b, cfg = cfg1_world
    u, v, t = w.get_state()
    a = w.assemble(u, t=t)
    s = oracle.Scene(b, cfg)
    ao = s.assemble(u, u, t=t, hess=False, pairs=True)
    assert a["n_pairs"][0] == ao["n_pairs"] > 0
    assert np.array_equal(w.contact_pairs(), ao["pairs"])
