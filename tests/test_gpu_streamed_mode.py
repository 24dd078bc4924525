"""The PCG's streamed-vector mode on small systems. When the CG vectors exceed half the L2 (the 1,024-body
batch), the update phase carries r in the preconditioned FP32 z and x as its FP64 value at the last
true-residual replacement plus an FP32 increment. Small systems use the exact FP64 vectors, so the other
tests do not reach that mode. Here the FP64-oracle parity tests and the executor test run again in a child
process with the mode forced on (SDX_PCG_R_IN_Z=1; the library reads the switch once per process), under
their own tolerances: vertex position within 1e-5 of the body size, Newton counts equal, CG counts within
max(6, 10 %)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_parity_with_r_and_x_carried_in_fp32():
    env = dict(os.environ, SDX_PCG_R_IN_Z="1")
    cmd = [sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider",
           os.path.join(HERE, "test_gpu_parity.py"),
           os.path.join(HERE, "test_gpu_snapshots.py") + "::test_executor_env_loop_with_resets_matches_fp64_oracle"]
    r = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "failed" not in r.stdout


def test_cluster_kernel_staged_update_phase():
    """The cluster kernel's update phase with its operands brought into shared memory by bulk asynchronous
    copies (what the 1,024-body batch runs): the cluster-batch tests again in a child process with z carrying
    r and the staging forced on (SDX_PCG_STAGE=1), against single-env steps and against the grid kernel."""
    env = dict(os.environ, SDX_PCG_R_IN_Z="1", SDX_PCG_STAGE="1")
    tests = os.path.join(HERE, "test_gpu_batch_repartition.py")
    cmd = [sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider",
           tests + "::test_cluster_batch_matches_single_env_steps",
           tests + "::test_cluster_and_grid_kernels_agree_on_a_contact_batch"]
    r = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "3 passed" in r.stdout
