"""sdx_pcg_solve_device_noalloc: the solve for callers that cannot allocate GPU memory when they need it
(an engine whose own pool allocator owns all device memory, a real-time loop that must not take
allocator locks). The caller owns every buffer (here: torch tensors standing in for the caller's pool);
the library's work vectors live in one fixed array inside the library. This file is collected last, so
a run that stops at its first failure has already run every other test; it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


def _fem_system(oracle, seed):
    """A projected Newton Hessian and gradient of a small heterogeneous tet grid."""
    rng = np.random.default_rng(seed)
    b = scenes.grid_body(7, 6, 5, 0.01, rng=rng, nu=0.45)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=b.n_tets))
    s = oracle.Scene(b, scenes.SceneConfig())
    u = rng.normal(0, 5e-4, 3 * b.n_nodes) * (b.pin == 0).repeat(3)
    a = s.assemble(u, u - 1e-4, psd=True)
    return s.row_ptr, s.col, a["H"].astype(np.float32), a["g"]


def _existing_entry_point(rp, col, H, b):
    from project_superdex_b200 import capi
    lp = capi.default_linear_params()
    lp.rel_tol = 1e-6
    st = capi.LinearStatus()
    x = np.zeros_like(b)
    Hc = np.ascontiguousarray(H)
    rc = capi.lib().sdx_pcg_solve(rp.size - 1, col.size, capi.ptr(rp, capi._lp), capi.ptr(col, capi._ip),
                                  Hc.ctypes.data_as(C.c_void_p), capi.SDX_F32, capi.ptr(b), capi.ptr(x),
                                  capi.SDX_GUESS_ZERO, C.byref(lp), C.byref(st))
    capi.check(rc)
    return x, st


def _no_alloc(rp, col, H, b):
    import torch
    from project_superdex_b200 import capi
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(np.ascontiguousarray(H).reshape(-1)).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.full_like(d_b, float("nan"))  # ignored for a zero initial guess
    lp = capi.default_linear_params()
    lp.rel_tol = 1e-6
    st = capi.LinearStatus()
    torch.cuda.synchronize()
    rc = capi.lib().sdx_pcg_solve_device_noalloc(rp.size - 1, col.size, d_rp.data_ptr(), d_col.data_ptr(),
                                                 d_val.data_ptr(), d_b.data_ptr(), d_x.data_ptr(),
                                                 capi.SDX_GUESS_ZERO, C.byref(lp), C.byref(st), None)
    capi.check(rc)
    return d_x.cpu().numpy(), st


def _true_rel_residual(rp, col, H, x, b):
    y = np.zeros_like(b)
    for i in range(rp.size - 1):
        for k in range(rp[i], rp[i + 1]):
            y[3 * i:3 * i + 3] += H[k].astype(np.float64) @ x[3 * col[k]:3 * col[k] + 3]
    return np.linalg.norm(b - y) / np.linalg.norm(b)


def test_no_alloc_matches_existing_entry_point_on_two_calls(oracle):
    systems = [_fem_system(oracle, 1), _fem_system(oracle, 2)]
    for rp, col, H, b in systems:  # two calls in a row: the shared array keeps the last call's contents
        x_ref, st_ref = _existing_entry_point(rp, col, H, b)
        x, st = _no_alloc(rp, col, H, b)
        assert st.convergence == st_ref.convergence == 1
        assert abs(st.num_iter - st_ref.num_iter) <= max(6, int(0.15 * st_ref.num_iter))
        assert _true_rel_residual(rp, col, H, x, b) <= 1.01e-6
        np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-4 * np.abs(x_ref).max())


def test_no_alloc_rejects_oversized_systems():
    from project_superdex_b200 import capi
    lp = capi.default_linear_params()
    st = capi.LinearStatus()
    n = capi.SDX_NOALLOC_MAX_BLOCK_ROWS + 1
    fake = 256  # never dereferenced: the size check comes first
    rc = capi.lib().sdx_pcg_solve_device_noalloc(n, 10, fake, fake, fake, fake, fake, capi.SDX_GUESS_ZERO,
                                                 C.byref(lp), C.byref(st), None)
    assert rc == -1
    assert b"65536" in capi.lib().sdx_last_error()
