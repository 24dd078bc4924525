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


def _params(prec=1, layout=None):
    from project_superdex_b200 import capi
    lp = capi.default_linear_params()
    lp.rel_tol = 1e-6
    lp.preconditioner = prec
    lp.value_layout = capi.SDX_BSR_BLOCKS if layout is None else layout
    return lp


def _existing_entry_point(rp, col, H, b, prec=1, x0=None):
    from project_superdex_b200 import capi
    lp = _params(prec)
    st = capi.LinearStatus()
    x = np.zeros_like(b) if x0 is None else x0.copy()
    Hc = np.ascontiguousarray(H)
    rc = capi.lib().sdx_pcg_solve(rp.size - 1, col.size, capi.ptr(rp, capi._lp), capi.ptr(col, capi._ip),
                                  Hc.ctypes.data_as(C.c_void_p), capi.SDX_F32, capi.ptr(b), capi.ptr(x),
                                  capi.SDX_GUESS_ZERO if x0 is None else capi.SDX_GUESS_UNKNOWN, C.byref(lp),
                                  C.byref(st))
    capi.check(rc)
    return x, st


class _DeviceSystem:
    """The caller's own device buffers (torch tensors standing in for the caller's pool)."""

    def __init__(self, rp, col, values, b, x0=None):
        import torch
        dev = torch.device("cuda:0")
        self.rp = torch.from_numpy(np.ascontiguousarray(rp)).to(dev)
        self.col = torch.from_numpy(np.ascontiguousarray(col)).to(dev)
        self.val = torch.from_numpy(np.ascontiguousarray(values).reshape(-1)).to(dev)
        self.b = torch.from_numpy(b).to(dev)
        self.x0 = None if x0 is None else torch.from_numpy(x0).to(dev)
        self.x = torch.full_like(self.b, float("nan"))  # ignored for a zero initial guess
        self.n, self.nnzb = int(rp.size - 1), int(col.size)
        torch.cuda.synchronize()

    def solve(self, lp):
        from project_superdex_b200 import capi
        if self.x0 is not None:
            self.x.copy_(self.x0)
        st = capi.LinearStatus()
        rc = capi.lib().sdx_pcg_solve_device_noalloc(self.n, self.nnzb, self.rp.data_ptr(), self.col.data_ptr(),
                                                     self.val.data_ptr(), self.b.data_ptr(), self.x.data_ptr(),
                                                     capi.SDX_GUESS_ZERO if self.x0 is None else capi.SDX_GUESS_UNKNOWN,
                                                     C.byref(lp), C.byref(st), None)
        return rc, st


def _no_alloc(rp, col, H, b, prec=1, x0=None):
    from project_superdex_b200 import capi
    d = _DeviceSystem(rp, col, H, b, x0)
    rc, st = d.solve(_params(prec))
    capi.check(rc)
    return d.x.cpu().numpy(), st


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


def test_no_alloc_block_jacobi_warm_start_and_reference_layout(oracle):
    """Block Jacobi, a supplied initial guess (InitialGuessHint::Unknown) and the reference's row-strip value
    layout give what sdx_pcg_solve gives."""
    from project_superdex_b200 import capi
    from project_superdex_b200.linear_solver import blocks_to_strips
    rp, col, H, b = _fem_system(oracle, 3)
    x_ref, st_ref = _existing_entry_point(rp, col, H, b, prec=2)
    x, st = _no_alloc(rp, col, H, b, prec=2)
    assert st.convergence == st_ref.convergence == 1
    assert abs(st.num_iter - st_ref.num_iter) <= max(6, int(0.15 * st_ref.num_iter))
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-4 * np.abs(x_ref).max())
    x0 = 0.9 * x_ref
    x_w, st_w = _existing_entry_point(rp, col, H, b, prec=1, x0=x0)
    x2, st2 = _no_alloc(rp, col, H, b, prec=1, x0=x0)
    assert st2.convergence == 1 and abs(st2.num_iter - st_w.num_iter) <= max(6, int(0.15 * st_w.num_iter))
    assert _true_rel_residual(rp, col, H, x2, b) <= 1.01e-6
    strips = blocks_to_strips(rp, H)
    d = _DeviceSystem(rp, col, strips, b)
    rc, st3 = d.solve(_params(1, capi.SDX_BSR_ROW_STRIPS))
    capi.check(rc)
    x3 = d.x.cpu().numpy()
    x1, st1 = _no_alloc(rp, col, H, b, prec=1)
    assert st3.num_iter == st1.num_iter and np.array_equal(x3, x1)


def test_no_alloc_allocates_nothing_on_a_second_call(oracle):
    """Free device memory is the same before and after a call once the one-time set-up has run."""
    import torch
    from project_superdex_b200 import capi
    rp, col, H, b = _fem_system(oracle, 4)
    d = _DeviceSystem(rp, col, H, b)
    lp = _params()
    rc, _ = d.solve(lp)  # set-up (symbol lookup) happens on the first call of the process, if not before
    capi.check(rc)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        rc, st = d.solve(lp)
        capi.check(rc)
        assert st.convergence == 1
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_no_alloc_rejects_a_malformed_row_ptr(oracle):
    """row_ptr not ending at nnzb, not monotone, or not starting at 0 is caught on the device before any
    load leaves the caller's arrays, and the call returns SDX_ERR_INVALID_ARGUMENT; a valid call after it
    converges."""
    from project_superdex_b200 import capi
    rp, col, H, b = _fem_system(oracle, 5)
    bad1 = rp.copy()
    bad1[-1] = rp[-1] + 7            # past nnzb
    bad2 = rp.copy()
    bad2[5], bad2[6] = rp[6], rp[5]  # not monotone
    bad3 = rp.copy()
    bad3[0] = 1                      # not starting at 0
    for bad in (bad1, bad2, bad3):
        d = _DeviceSystem(bad, col, H, b)
        rc, _ = d.solve(_params())
        assert rc == capi.SDX_ERR_INVALID_ARGUMENT, rc
        assert b"row_ptr" in capi.lib().sdx_last_error()
    x, st = _no_alloc(rp, col, H, b)
    assert st.convergence == 1 and _true_rel_residual(rp, col, H, x, b) <= 1.01e-6


def test_bounded_device_waits_time_out_and_recover(oracle, monkeypatch):
    """With the spin bound lowered to a few polls (SDX_DEBUG_SPIN_LIMIT), the grid barriers of the
    no-allocation kernel and of the context PCG give up: both calls return SDX_ERR_DEVICE_TIMEOUT and the
    kernels unwind. The next calls with the normal bound converge (the barrier words are reset per call)."""
    from project_superdex_b200 import capi
    rp, col, H, b = _fem_system(oracle, 6)
    d = _DeviceSystem(rp, col, H, b)
    monkeypatch.setenv("SDX_DEBUG_SPIN_LIMIT", "2")
    rc, _ = d.solve(_params())
    assert rc == capi.SDX_ERR_DEVICE_TIMEOUT, rc
    with pytest.raises(capi.SdxError, match="sdx error -4"):
        _existing_entry_point(rp, col, H, b)
    monkeypatch.delenv("SDX_DEBUG_SPIN_LIMIT")
    rc, st = d.solve(_params())
    capi.check(rc)
    assert st.convergence == 1
    x, st2 = _existing_entry_point(rp, col, H, b)
    assert st2.convergence == 1 and _true_rel_residual(rp, col, H, x, b) <= 1.01e-6


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
