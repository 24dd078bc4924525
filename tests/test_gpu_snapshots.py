"""State snapshots (device-resident capture / restore, the bytes format, per-env restore), masked state
writes and the batched executor's step-and-readback loop, as the reference's Scene state API and
SceneBatchExecutorV2 define them (mochi_scene.h:79-93, scene_batch_executor_v2.cpp:335-745) and as the
Lab environments use them around every environment step (mochi_env.py:786-821)."""
import numpy as np
import pytest

from project_superdex_b200 import capi, scenes
from project_superdex_b200.executor import READ_CONTACTS, READ_DIVERGED, READ_QPOS, READ_QVEL, SoftSceneBatchExecutor

pytestmark = pytest.mark.gpu

SIZE = 0.05
# Two runs of the same steps differ by the rounding order of the assembly's atomic accumulation, which the
# Newton and CG solves carry up to their tolerances (observed ~1e-11 m here); the oracle-parity bar is 1e-5.
TOL = 1e-8 * SIZE


def _bodies(seed=3, dims=((4, 4, 4), (5, 3, 4), (3, 4, 5))):
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny, nz in dims:
        b = scenes.grid_body(nx, ny, nz, 0.01, rng=rng, E=float(rng.uniform(5e4, 3e5)), nu=0.4)
        top = nz * 0.01
        b.colliders = [scenes.capsule((0.01, 0.01, top + 0.0035), (0.03, 0.02, top + 0.0035), 0.004,
                                      (0.02, 0.0, -0.15))]
        out.append(b)
    return out


def _world(bodies=None, **kw):
    from project_superdex_b200.soft_body import SoftBodyWorld
    cfg = scenes.SceneConfig(k_contact=1e6, friction_coulomb=0.5)
    return SoftBodyWorld(bodies if bodies is not None else _bodies(), cfg, warm_start=capi.SDX_WARM_TEMPORAL, **kw)


def test_restore_then_step_repeats_the_trajectory():
    w = _world()
    w.step(2)
    h = w.capture_state()
    w.step(3)
    ua, va, ta = w.get_state()
    sa = w.stats()
    w.restore_state(h)
    assert w.get_state()[2] == pytest.approx(ta - 3 * w.params.dt)
    w.step(3)
    ub, vb, tb = w.get_state()
    assert tb == ta
    assert np.abs(ua - ub).max() <= TOL
    assert np.abs(va - vb).max() <= TOL / w.params.dt
    for x, y in zip(sa, w.stats()):
        assert x["newton_iters"] == y["newton_iters"]
        assert abs(x["cg_iters"] - y["cg_iters"]) <= 2
    w.close()


def test_bytes_round_trip_into_a_fresh_context():
    bodies = _bodies()
    w1 = _world(bodies)
    w1.step(2)
    u0, v0, t0 = w1.get_state()
    blob = w1.capture_state_to_bytes()
    w1.step(2)
    u1, _, _ = w1.get_state()
    w2 = _world(bodies)
    w2.restore_state_from_bytes(blob)
    u, v, t = w2.get_state()
    assert t == t0 and np.array_equal(u, u0) and np.array_equal(v, v0)  # the exact state, bit for bit
    assert w2.capture_state_to_bytes() == blob
    w2.step(2)
    assert np.abs(w2.get_state()[0] - u1).max() <= TOL
    w1.close()
    w2.close()


def test_bytes_are_refused_for_other_bodies_or_when_damaged():
    w = _world()
    w.step(1)
    blob = bytearray(w.capture_state_to_bytes())
    other = _world(_bodies(seed=4))
    with pytest.raises(capi.SdxError, match="different bodies"):
        other.restore_state_from_bytes(bytes(blob))
    bad = bytearray(blob)
    bad[len(bad) // 2] ^= 0x40
    with pytest.raises(capi.SdxError, match="checksum"):
        w.restore_state_from_bytes(bytes(bad))
    with pytest.raises(capi.SdxError):
        w.restore_state_from_bytes(bytes(blob[:-9]))
    with pytest.raises(capi.SdxError, match="not a state snapshot"):
        w.restore_state_from_bytes(b"\0" * 64)
    w.close()
    other.close()


def test_per_env_restore_and_masked_writes():
    w = _world()
    off = w.node_off
    w.step(1)
    h = w.capture_state()
    u_snap, v_snap, _ = w.get_state()
    w.step(2)
    u_now, v_now, t_now = w.get_state()
    w.restore_state(h, env_mask=np.array([0, 1, 0], np.uint8))
    u, v, t = w.get_state()
    assert t == t_now  # the clock is shared by the envs and stays
    sl = [slice(3 * off[e], 3 * off[e + 1]) for e in range(3)]
    assert np.array_equal(u[sl[1]], u_snap[sl[1]]) and np.array_equal(v[sl[1]], v_snap[sl[1]])
    for e in (0, 2):
        assert np.array_equal(u[sl[e]], u_now[sl[e]]) and np.array_equal(v[sl[e]], v_now[sl[e]])
    # masked write: z displacement of env 2 only
    q = np.full(u.size, 1e-3)
    mask = np.zeros(u.size, np.uint8)
    mask[sl[2]][2::3] = 1
    w.write_state(qpos=q, qpos_write_mask=mask)
    u2, v2, _ = w.get_state()
    want = u.copy()
    want[mask.astype(bool)] = 1e-3
    assert np.array_equal(u2, want) and np.array_equal(v2, v)
    w.close()


def test_snapshot_equality_release_and_unknown_handles():
    w = _world()
    w.step(1)
    a = w.capture_state()
    b = w.capture_state()
    assert w.is_equal_state(a, b)
    w.step(1)
    c = w.capture_state()
    assert not w.is_equal_state(a, c)
    w.release_state(b)
    w.release_state(b)  # redundant releases are ignored
    assert not w.is_equal_state(a, b)
    with pytest.raises(capi.SdxError, match="invalid state handle"):
        w.restore_state(b)
    w.restore_state(a, release_immediately=True)
    with pytest.raises(capi.SdxError, match="invalid state handle"):
        w.restore_state(a)
    other = _world()
    with pytest.raises(capi.SdxError, match="invalid state handle"):
        other.restore_state(c)  # a handle of another context
    w.release_all_states()
    with pytest.raises(capi.SdxError):
        w.restore_state(c)
    w.close()
    other.close()


def test_executor_env_loop_matches_plain_stepping():
    """The Lab environment pattern: restore the env-step snapshot (released at once), step, read back the
    selected outputs, capture the next snapshot; the trajectory is plain stepping's."""
    ref = _world()
    ref.step(4)
    u_ref, v_ref, _ = ref.get_state()
    with SoftSceneBatchExecutor(_world()) as ex:
        n, s = ex.num_dofs, ex.num_scenes
        assert ex.scene_dof_offsets[-1] == n and s == 3
        qpos, qvel = np.zeros(n), np.zeros(n)
        contacts, diverged = np.zeros(s), np.ones(s, np.uint8)
        snap = None
        for _ in range(4):
            if snap is not None:
                ex.restore_state(snap, release_immediately=True)
            ex.step(ex.world.params.dt, None, qpos, qvel, None, contacts, diverged,
                    READ_QPOS | READ_QVEL | READ_CONTACTS | READ_DIVERGED)
            snap = ex.capture_state()
        u, v, _ = ex.world.get_state()
        assert np.array_equal(qpos, u) and np.array_equal(qvel, v)
        assert np.abs(u - u_ref).max() <= TOL
        assert np.array_equal(contacts, [st["n_contacts"] for st in ex.world.stats()]) and contacts.max() > 0
        assert not diverged.any()
        only_q = np.zeros(n)
        ex.step(ex.world.params.dt, np.zeros(n), only_q, None, None, None, None, READ_QPOS)
        assert np.array_equal(only_q, ex.world.get_state()[0])
        with pytest.raises(ValueError):
            ex.step(ex.world.params.dt, np.ones(n), only_q, None, None, None, None, READ_QPOS)
    assert ex.closed
    with pytest.raises(RuntimeError):
        ex.step(1 / 240.0)
    ref.close()


def test_executor_env_loop_with_resets_matches_fp64_oracle(oracle):
    """The Lab loop (mochi_env.py:786-821) over SoftSceneBatchExecutor against the FP64 CPU oracle stepping
    the same sequence per env: restore the env-step snapshot, step, read back, capture; then a batched
    reset of env 1 to an earlier snapshot (per-env restore, the clock kept) and more steps. Every env's
    displacement after every step is within 1e-5 of the body size of the oracle's."""
    bodies = _bodies()
    cfg = scenes.SceneConfig(k_contact=1e6, friction_coulomb=0.5)
    sc = [oracle.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps)) for b in bodies]
    p = oracle.default_newton_params()
    ost = [(np.zeros(3 * b.n_nodes), np.zeros(3 * b.n_nodes)) for b in bodies]
    off = np.concatenate([[0], np.cumsum([3 * b.n_nodes for b in bodies])])
    dt = cfg.dt
    with SoftSceneBatchExecutor(_world(bodies)) as ex:
        n = ex.num_dofs
        qpos, qvel = np.zeros(n), np.zeros(n)
        snap, saved, saved_oracle = None, None, None
        for k in range(7):
            if k == 5:  # batched reset: env 1 back to its state after step 3, the others go on
                ex.world.restore_state(saved, env_mask=np.array([0, 1, 0], np.uint8))
                ost[1] = saved_oracle
            elif snap is not None:
                ex.restore_state(snap, release_immediately=True)
            ex.step(dt, None, qpos, qvel, None, None, None, READ_QPOS | READ_QVEL)
            snap = ex.capture_state()
            if k == 2:
                saved = ex.capture_state()
            t = (k + 1) * dt  # the world clock (a per-env restore keeps it)
            for e in range(3):
                u, v, st = sc[e].step(ost[e][0], ost[e][1], t, p)
                ost[e] = (u, v)
                err = np.abs(qpos[off[e]:off[e + 1]] - u).max()
                assert err <= 1e-5 * SIZE, (k, e, err)
            if k == 2:
                saved_oracle = (ost[1][0].copy(), ost[1][1].copy())
        st = ex.world.stats()
        assert all(s["convergence"] == 1 for s in st) and max(s["n_contacts"] for s in st) > 0
