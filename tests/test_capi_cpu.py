"""The C-ABI library: loads, exports every entry point include/sdx_b200.h declares, and its structs agree
with the Python mirror. No compute call runs here (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sdx_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sdx_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from project_superdex_b200 import capi
    lib = capi.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/sdx_b200.h but not exported"
    assert set(names) == set(capi.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sdx_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_struct_layouts_match_header(tmp_path):
    from project_superdex_b200 import capi
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "sdx_b200.h"\nint main(){printf("%zu %zu %zu %zu %zu %zu\\n",'
                   'sizeof(sdx_linear_params),sizeof(sdx_linear_status),sizeof(sdx_step_params),sizeof(sdx_env_stats),'
                   'sizeof(sdx_profile),offsetof(sdx_step_params,linear));return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.check_call(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    want = [C.sizeof(capi.LinearParams), C.sizeof(capi.LinearStatus), C.sizeof(capi.StepParams),
            C.sizeof(capi.EnvStats), C.sizeof(capi.Profile), capi.StepParams.linear.offset]
    assert got == want


def test_defaults_mirror_reference_defaults():
    from project_superdex_b200 import capi
    p = capi.default_step_params()
    assert p.ls_max_iter == 4 and p.ls_alpha == 0.5  # nonlinear_solver_params.h:417-424
    assert p.rel_div_tol == 1e4 and p.abs_div_tol == 1e9  # :400-408
    assert p.newton_rel_tol == 1e-6 and p.newton_abs_tol == 1e-3  # :361-364
    assert p.k_contact == 1e9 and p.t_half == 0.005 and p.thr == 0.001  # contact_params.h:96-123
    assert p.psd_strategy == capi.SDX_PSD_PROJECTION if hasattr(capi, "SDX_PSD_PROJECTION") else p.psd_strategy == 1
    lp = capi.default_linear_params()
    assert lp.abs_tol == 1e-9 and lp.rel_div_tol == 1e10 and lp.polak_ribiere == 1 and lp.preconditioner == 1
    # the options with no counterpart in the reference are off by default: a plain unrestarted PCG and a
    # host-driven Newton loop, as the reference runs them
    assert lp.refine_inner_rel_tol == 0.0 and lp.refine_max_passes == 8
    assert p.newton_graph == 0 and p.linear.refine_inner_rel_tol == 0.0 and p.warm_start == capi.SDX_WARM_ZERO


def test_no_gpu_is_reported_not_faked():
    """Without a device the library refuses to create a context (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from project_superdex_b200 import capi
    lib = capi.lib()
    assert not lib.sdx_create(0)
    assert b"device" in lib.sdx_last_error().lower() or b"cuda" in lib.sdx_last_error().lower()
    with pytest.raises(capi.SdxError, match="no CUDA device"):
        capi.pcg_cluster_shape(16)  # the cluster PCG's launch shape needs the device it would run on


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from project_superdex_b200 import capi
    monkeypatch.setattr(capi, "_lib", None)
    monkeypatch.setattr(capi, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        capi.lib()


def test_product_library_links_no_second_solver_backend():
    """libsdx_b200.so has one linear solver: the cuSPARSE / cuBLAS comparison arm lives in the benchmark's
    own library (bench_arms/libsdx_plain_fp64.so), plugged in through sdx_set_linear_solver."""
    from project_superdex_b200 import capi
    deps = subprocess.run(["ldd", capi.LIB_PATH], capture_output=True, text=True).stdout
    assert "cusparse" not in deps and "cublas" not in deps
    plain = os.path.join(ROOT, "bench_arms", "libsdx_plain_fp64.so")
    if os.path.exists(plain):
        out = subprocess.run(["nm", "-D", "--defined-only", plain], capture_output=True, text=True).stdout
        for sym in ("sdx_plain_fp64_create", "sdx_plain_fp64_destroy", "sdx_plain_fp64_solve"):
            assert f" T {sym}" in out
