"""The per-warp TMA-ring operator (FP32 edge records): points with more than
32 observations (tiles of their own), the global camera accumulator used when
the camera sums do not fit one SM's shared memory, and the bounded slot wait,
all checked against the oracle's reduced operator and steps
(src/schur.rs:596-652, 204-344)."""
import dataclasses

import numpy as np
import pytest

import fagra_b200 as fg
import oracle
from fagra_b200 import synthetic

pytestmark = pytest.mark.gpu


def deep_problem(cameras=64, points=3000, deep=(0, 1, 2, 1500, 2999), seed=9):
    """A bal1k-shaped problem whose `deep` points are seen by every camera."""
    d = synthetic.generate("bal1k", cameras=cameras, points=points, seed=seed)
    add_c, add_p = [], []
    for p in deep:
        have = set(d.obs_camera[d.obs_point == p].tolist())
        for c in range(cameras):
            if c not in have:
                add_c.append(c)
                add_p.append(p)
    ac, ap = np.array(add_c, np.uint32), np.array(add_p, np.uint32)
    pix, depth = synthetic.project(d.true_cameras, d.true_points, ac, ap)
    assert np.all(depth < 0)
    px = pix + 0.5 * np.random.default_rng(seed).normal(size=pix.shape)
    return dataclasses.replace(d, obs_camera=np.concatenate([d.obs_camera, ac]),
                               obs_point=np.concatenate([d.obs_point, ap]),
                               obs_pixel=np.concatenate([d.obs_pixel, px]))


def _oracle(d, lam=None, x=None):
    o = oracle.Schur(9 * d.num_cameras, 9, 3)
    ob = oracle.Bal.from_data(d)
    o.prepare(ob.dimension())
    ob.linearize(o)
    o.prepare_damping(1e-6)
    return o


def _device(d, precision="f32", **kw):
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision=precision, **kw)
    p = fg.BalProblem.from_data(d)
    b.prepare(p.dimension())
    p.linearize(b)
    b.prepare_damping(1e-6)
    return b, p


@pytest.mark.parametrize("lam", [1e-3, 1.0])
def test_ring_operator_with_deep_points_matches_oracle(lam):
    d = deep_problem()
    counts = np.bincount(d.obs_point, minlength=d.num_points)
    assert counts.max() > 32
    o = _oracle(d)
    b, _ = _device(d)
    assert b.operator_info()[0] == 1  # deep points leave only the ring kernel
    x = np.random.default_rng(3).normal(size=9 * d.num_cameras)
    ref = o.reduced_apply(lam, x)
    got = b.reduced_apply(lam, x)
    assert np.linalg.norm(got - ref) <= 2e-5 * np.linalg.norm(ref)


def test_ring_steps_with_deep_points_match_oracle():
    """Right-hand side, PCG and point back-substitution through the ring
    kernel: the FP32 step equals the oracle's f64 step to FP32 accuracy and
    the reduced residual is below 1e-8."""
    d = deep_problem()
    o = _oracle(d)
    _, ref, pred = o.solve_damped(1e-3)
    for coarse in (False, True):
        b, _ = _device(d, coarse_correction=coarse)
        b.relative_tolerance = 1e-10
        st = b.solve_damped(1e-3)
        assert b.diagnostics().reduced_relative_residual < 1e-8
        assert np.linalg.norm(st.delta - ref) <= 1e-4 * np.linalg.norm(ref), coarse
        assert abs(st.predicted_reduction - pred) <= 1e-6 * abs(pred)


def test_ring_lm_with_deep_points_reaches_oracle_cost():
    d = deep_problem()
    code, rep, st = oracle.Bal.from_data(d).lm(oracle.Schur(9 * d.num_cameras, 9, 3), max_iterations=20)
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision="f32", coarse_correction=True)
    b.relative_tolerance = 1e-8
    out = fg.LevenbergMarquardt(b).solve_batch_with_outcome(fg.BalProblem.from_data(d),
                                                             fg.OptimizeOptions(20, 1e-8, 0.0, 0.0))
    assert abs(out.statistics.cost - st.cost) <= 1e-6 * st.cost


@pytest.mark.parametrize("lam", [1e-3, 1.0])
def test_ring_global_accumulator_matches_oracle(lam):
    """3,000 cameras: the operator's fixed-point camera sums (72 bytes per
    camera) and the slots (74 KB) no longer fit one SM's shared memory, so the
    camera sums go to the global accumulator (FP32 vector reductions into 8
    copies, summed in FP64)."""
    d = synthetic.generate("bal1k", cameras=3000, points=30000, seed=11)
    o = _oracle(d)
    b, _ = _device(d)
    assert b.operator_info()[0] == 1
    x = np.random.default_rng(5).normal(size=9 * d.num_cameras)
    ref = o.reduced_apply(lam, x)
    got = b.reduced_apply(lam, x)
    assert np.linalg.norm(got - ref) <= 2e-5 * np.linalg.norm(ref)
    # the accumulator is cleared by each reduction: a second application agrees
    again = b.reduced_apply(lam, x)
    assert np.linalg.norm(again - got) <= 1e-6 * np.linalg.norm(ref)


def test_ring_global_accumulator_steps_match_oracle():
    d = synthetic.generate("bal1k", cameras=3000, points=30000, seed=11)
    o = _oracle(d)
    _, ref, pred = o.solve_damped(1e-3)
    for coarse in (False, True):
        b, _ = _device(d, coarse_correction=coarse)
        b.relative_tolerance = 1e-10
        st = b.solve_damped(1e-3)
        assert b.diagnostics().reduced_relative_residual < 1e-8
        assert np.linalg.norm(st.delta - ref) <= 1e-4 * np.linalg.norm(ref), coarse
        assert abs(st.predicted_reduction - pred) <= 1e-6 * abs(pred)


def test_ring_slot_wait_times_out_then_recovers():
    """With the consumer wait limited to one poll the slot wait gives up, the
    kernel drains its copies in flight and the solve returns
    FG_DEVICE_TIMEOUT; with the default limit the next solve succeeds and
    gives the normal step. No fault: the copies complete, only the wait is
    cut short."""
    d = synthetic.generate("bal16")
    ref_b, _ = _device(d)
    ref = ref_b.solve_damped(1e-3).delta.copy()
    b, _ = _device(d)
    b.set_poll_limit(1)
    with pytest.raises(fg.DeviceTimeout):
        b.solve_damped(1e-3)
    b.set_poll_limit(0)
    got = b.solve_damped(1e-3).delta
    assert np.linalg.norm(got - ref) <= 1e-6 * np.linalg.norm(ref)


@pytest.mark.parametrize("lam", [1e-3, 1.0])
def test_ring_fixed_point_sums_of_high_degree_cameras(lam):
    """16 cameras seeing 40,000 points four times each: every camera holds
    about 10,000 observations, so each CTA adds hundreds of contributions into
    a camera's 64-bit fixed-point sums; the FP32-record operator matches the
    f64-record operator and the oracle to FP32 accuracy."""
    d = synthetic.generate("bal16", points=40_000, seed=3)
    counts = np.bincount(d.obs_camera, minlength=d.num_cameras)
    assert counts.min() > 9_000
    o = _oracle(d)
    b32, _ = _device(d)
    assert b32.operator_info()[0] == 1
    b64, _ = _device(d, precision="f64")
    x = np.random.default_rng(7).normal(size=9 * d.num_cameras)
    ref = o.reduced_apply(lam, x)
    got32, got64 = b32.reduced_apply(lam, x), b64.reduced_apply(lam, x)
    assert np.linalg.norm(got64 - ref) <= 1e-10 * np.linalg.norm(ref)
    assert np.linalg.norm(got32 - got64) <= 2e-5 * np.linalg.norm(got64)
