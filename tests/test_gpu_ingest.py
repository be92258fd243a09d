"""Device ingestion of BAL problems: observations in any insertion order are
validated, put in emission order (one Frame batch per camera, insertion order
within, examples/bal/model.rs:187-200) and turned into the Schur structure by
device radix orders; checked against numpy's stable orders and a numpy
restatement of the gradient J^T r on problems whose point indices need
several radix passes."""
import dataclasses

import numpy as np
import pytest

import fagra_b200 as fg
from fagra_b200 import synthetic

pytestmark = pytest.mark.gpu


def _shuffled(d, seed):
    perm = np.random.default_rng(seed).permutation(d.num_observations)
    return dataclasses.replace(d, obs_camera=d.obs_camera[perm].copy(), obs_point=d.obs_point[perm].copy(),
                               obs_pixel=d.obs_pixel[perm].copy())


def _linearized(d):
    b = fg.Schur(9 * d.num_cameras, 9, 3)
    p = fg.BalProblem.from_data(d)
    b.prepare(p.dimension())
    p.linearize(b)
    b.prepare_damping(1e-6)
    return b, p


@pytest.mark.parametrize("cameras,points", [(40, 3000), (64, 70000)])
def test_emission_order_and_gradient_of_shuffled_observations(cameras, points):
    d = _shuffled(synthetic.generate("bal1k", cameras=cameras, points=points, seed=7), seed=points)
    b, _ = _linearized(d)
    s, m = b.structure(), b.model()
    order = np.argsort(d.obs_camera, kind="stable")
    cam, pt = d.obs_camera[order].astype(np.int64), d.obs_point[order].astype(np.int64)
    k = np.arange(d.num_observations)
    want = np.zeros((2 * len(k), 5), np.int64)
    want[0::2] = np.stack([2 * k, 9 * cam, np.full_like(k, 2), np.full_like(k, 9), 24 * k], 1)
    want[1::2] = np.stack([2 * k, 9 * cameras + 3 * pt, np.full_like(k, 2), np.full_like(k, 3), 24 * k + 18], 1)
    assert np.array_equal(s["blocks"].astype(np.int64), want)
    assert np.array_equal(s["edges"][:, :2].astype(np.int64), np.stack([9 * cam, 3 * pt], 1))
    # gradient J^T r from the emitted blocks (each block column-major, 2 rows)
    vals, r = m["values"].reshape(-1, 24), -m["negative_residual"].reshape(-1, 2)
    Jc = vals[:, :18].reshape(-1, 9, 2)  # [emission, column, row]
    Jp = vals[:, 18:].reshape(-1, 3, 2)
    g = np.zeros(d.dimension())
    np.add.at(g, (9 * cam)[:, None] + np.arange(9), np.einsum("ecr,er->ec", Jc, r))
    np.add.at(g, (9 * cameras + 3 * pt)[:, None] + np.arange(3), np.einsum("ecr,er->ec", Jp, r))
    assert np.max(np.abs(m["gradient"] - g)) <= 1e-10 * np.max(np.abs(g))


def test_insertion_orders_with_equal_frames_give_equal_models():
    # two insertion orders with the same per-camera order give the same model
    d = synthetic.generate("bal1k", cameras=40, points=3000, seed=3)
    a, _ = _linearized(d)
    order = np.argsort(d.obs_camera, kind="stable")
    e = dataclasses.replace(d, obs_camera=d.obs_camera[order].copy(), obs_point=d.obs_point[order].copy(),
                            obs_pixel=d.obs_pixel[order].copy())
    b, _ = _linearized(e)
    ma, mb = a.model(), b.model()
    for key in ("values", "negative_residual", "gradient", "scales", "gram", "cross"):
        assert np.array_equal(ma[key], mb[key]), key


@pytest.mark.parametrize("fault", ["camera", "point", "pixel"])
def test_invalid_observations_are_rejected(fault):
    d = synthetic.generate("bal16")
    oc, op, px = d.obs_camera.copy(), d.obs_point.copy(), d.obs_pixel.copy()
    i = len(oc) // 2
    if fault == "camera":
        oc[i] = d.num_cameras
    elif fault == "point":
        op[i] = d.num_points + 5
    else:
        px[i, 1] = np.nan
    with pytest.raises(fg.errors.InvalidEmission):
        fg.BalProblem(d.cameras, d.points, oc, op, px)
    # the device stays usable and the next problem is ingested normally
    p = fg.BalProblem.from_data(d)
    assert np.isfinite(p.cost())


def test_parameters_into_caller_arrays():
    d = synthetic.generate("bal16")
    p = fg.BalProblem.from_data(d)
    c0, p0 = p.parameters()
    out = (np.full((d.num_cameras, 9), np.nan), np.full((d.num_points, 3), np.nan))
    c1, p1 = p.parameters(out=out)
    assert c1 is out[0] and p1 is out[1]
    assert np.array_equal(c0, c1) and np.array_equal(p0, p1) and np.array_equal(c0, d.cameras)
    with pytest.raises(ValueError):
        p.parameters(out=(np.zeros((d.num_cameras, 9), np.float32), out[1]))


def test_bal_text_file_end_to_end(tmp_path):
    """A problem written in the BAL text format (examples/bal/model.rs:58-114)
    and read back with synthetic.parse_bal (exactly: every value round-trips)
    runs through device ingestion and LM like the in-memory problem it was
    written from."""
    d = synthetic.generate("bal16", points=600, seed=4)
    lines = [f"{d.num_cameras} {d.num_points} {d.num_observations}"]
    lines += [f"{int(c)} {int(p)} {float(x)!r} {float(y)!r}" for c, p, (x, y) in zip(d.obs_camera, d.obs_point,
                                                                                   d.obs_pixel)]
    lines += [repr(float(v)) for v in d.cameras.reshape(-1)]
    lines += [repr(float(v)) for v in d.points.reshape(-1)]
    path = tmp_path / "problem.txt"
    path.write_text("\n".join(lines) + "\n")
    cams, pts, oc, op, px = synthetic.parse_bal(path.read_text())
    assert np.array_equal(cams, d.cameras) and np.array_equal(pts, d.points)
    assert np.array_equal(px, d.obs_pixel)
    opts = fg.OptimizeOptions(max_iterations=6)
    runs = []
    for prob in (fg.BalProblem(cams, pts, oc, op, px), fg.BalProblem.from_data(d)):
        lm = fg.LevenbergMarquardt(fg.Schur(9 * d.num_cameras, 9, 3))
        out = lm.solve_batch_with_outcome(prob, opts)
        runs.append((out.statistics.cost, out.statistics.accepted_steps, prob.parameters()))
    # the same inputs; the f64 operator's shared FP64 atomics may round in a different order
    assert abs(runs[0][0] - runs[1][0]) <= 1e-12 * runs[1][0] and runs[0][1] == runs[1][1]
    for a, b in zip(runs[0][2], runs[1][2]):
        assert np.allclose(a, b, rtol=1e-9, atol=1e-12)
