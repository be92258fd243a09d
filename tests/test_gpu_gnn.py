"""Learned preconditioner on the device against the oracle (oracle/gnn.py):
features, covisibility and probes of captured reduced camera systems, the BF16
tensor-core forward and backward passes, training, and the learned PCG with
its block-Jacobi fallback."""
import numpy as np
import pytest

import fagra_b200 as fg
from fagra_b200 import synthetic
from oracle import gnn as og

pytestmark = pytest.mark.gpu


def _random_system(C, seed, K=4, cw=9):
    rng = np.random.default_rng(seed)
    X0 = (rng.normal(size=(C, og.FEATURES)) * 0.5).astype(np.float32)
    W = np.abs(rng.normal(size=(C, C)))
    W = W + W.T
    np.fill_diagonal(W, 0.0)
    W[W < 1.0] = 0.0
    rows = W.sum(1)
    A = np.where(rows[:, None] > 0, W / np.where(rows > 0, rows, 1)[:, None], 0.0).astype(np.float32)
    X = rng.normal(size=(K, C, cw)).astype(np.float32)
    Y = (X + 0.3 * rng.normal(size=(K, C, cw))).astype(np.float32)
    mask = (rng.random(C) > 0.1).astype(np.uint8)
    return X0, A, X, Y, mask


def _random_parameters(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=n) * 0.15).astype(np.float32)


@pytest.mark.parametrize("C", [37, 300])
def test_forward_and_gradient_match_oracle(C):
    net = fg.LearnedPreconditioner(seed=3)
    flat = _random_parameters(net.parameter_count(), C)
    net.set_parameters(flat)
    idx = net.import_system(*_random_system(C, seed=C))
    s = net.export_system(idx)  # the device copy: adjacency rounded to bf16
    loss, g, out = net.evaluate(idx, gradient=True)
    ref_loss, ref_g, ref_out = og.loss_and_gradient(flat.astype(np.float64), s["features"], s["adjacency"],
                                                     s["probe_x"], s["probe_y"], s["mask"].astype(bool), 9,
                                                     rounded=True)
    assert np.linalg.norm(out - ref_out) <= 1e-3 * np.linalg.norm(ref_out)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    offsets = np.cumsum([0] + [int(np.prod(sh)) for _, sh in og.layout()])
    for k, (name, _) in enumerate(og.layout()):
        a, b = g[offsets[k]:offsets[k + 1]], ref_g[offsets[k]:offsets[k + 1]]
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-9, name


def _bal_backend(data, precision="f64", preconditioner="retained_blocks", damping_floor=1e-6):
    b = fg.Schur(9 * data.num_cameras, 9, 3, precision=precision, preconditioner=preconditioner)
    p = fg.BalProblem.from_data(data)
    b.prepare(p.dimension())
    p.linearize(b)
    b.prepare_damping(damping_floor)
    return b, p


def _sym_lower(v, w):
    m = v.reshape(w, w).T  # column major: element (r, c) at c*w + r
    return np.tril(m) + np.tril(m, -1).T


def _oracle_inputs(backend):
    s, m = backend.structure(), backend.model()
    cw, pw = backend.widths
    nC = backend.retained // cw
    nP = (s["cols"] - backend.retained) // pw
    cam_gram, pt_gram = np.zeros((nC, cw, cw)), np.zeros((nP, pw, pw))
    cam_obs, pt_obs = np.zeros(nC, bool), np.zeros(nP, bool)
    for col, w, start in s["variables"].astype(np.int64):
        blk = _sym_lower(m["gram"][start:start + w * w], w)
        if col < backend.retained:
            cam_gram[col // cw], cam_obs[col // cw] = blk, True
        else:
            q = (col - backend.retained) // pw
            pt_gram[q], pt_obs[q] = blk, True
    edges = np.stack([s["edges"][:, 0] // cw, s["edges"][:, 1] // pw], 1).astype(np.int64)
    cross = m["cross"].reshape(-1, pw, cw).transpose(0, 2, 1)
    return cam_gram, pt_gram, edges, cross, cam_obs, pt_obs


def test_captured_features_covisibility_and_probes_match_oracle():
    d = synthetic.generate("bal16")
    b, _ = _bal_backend(d)
    net = fg.LearnedPreconditioner(seed=1)
    lam = 3e-3
    idx = net.capture(b, lam, probes=3, seed=7, kind="products")
    s = net.export_system(idx)
    X0, A, Lc = og.system_features(*_oracle_inputs(b), lam)
    assert s["damping"] == lam and s["mask"].all()
    assert np.max(np.abs(s["features"] - X0)) <= 1e-5 * max(1.0, np.max(np.abs(X0)))
    assert np.max(np.abs(s["adjacency"] - og.bf16(A))) <= 2.0 ** -8 * np.max(A)
    # probes: y_hat = L^-1 S L^-T x_hat with S applied by the backend in f64
    for k in range(3):
        xh = s["probe_x"][k].astype(np.float64)
        x = np.concatenate([np.linalg.solve(Lc[i].T, xh[i]) for i in range(len(Lc))])
        y = b.reduced_apply(lam, x).reshape(-1, 9)
        yh = np.stack([np.linalg.solve(Lc[i], y[i]) for i in range(len(Lc))])
        assert np.linalg.norm(s["probe_y"][k] - yh) <= 1e-5 * np.linalg.norm(yh)
        assert abs(np.mean(xh)) < 0.2 and 0.7 < np.std(xh) < 1.3


def test_solve_probes_invert_the_whitened_system():
    d = synthetic.generate("bal16")
    b, _ = _bal_backend(d)
    net = fg.LearnedPreconditioner(seed=1)
    lam = 1e-2
    idx = net.capture(b, lam, probes=2, seed=3, kind="solves")
    s = net.export_system(idx)
    _, _, Lc = og.system_features(*_oracle_inputs(b), lam)
    for k in range(2):
        xh = s["probe_x"][k].astype(np.float64)
        x = np.concatenate([np.linalg.solve(Lc[i].T, xh[i]) for i in range(len(Lc))])
        y = b.reduced_apply(lam, x).reshape(-1, 9)
        yh = np.stack([np.linalg.solve(Lc[i], y[i]) for i in range(len(Lc))])
        assert np.linalg.norm(yh - s["probe_y"][k]) <= 1e-5 * np.linalg.norm(s["probe_y"][k])
    assert b.statistics().solves == 0  # probe solves leave the work counters alone


def test_untrained_network_is_block_jacobi():
    d = synthetic.generate("bal16")
    ref, _ = _bal_backend(d)
    step_bj = ref.solve_damped(1e-2).delta
    its_bj = ref.diagnostics().iterations
    b, _ = _bal_backend(d, preconditioner="learned")
    net = fg.LearnedPreconditioner(seed=2)
    b.attach_learned(net)
    step = b.solve_damped(1e-2).delta
    di = b.diagnostics()
    assert di.learned_iterations > 0 and di.block_jacobi_iterations == its_bj
    assert abs(di.learned_iterations - its_bj) <= 1
    assert di.learned_fallback in (None, "more_iterations")
    assert np.linalg.norm(step - step_bj) <= 1e-8 * np.linalg.norm(step_bj)


def _held_out():
    return synthetic.generate("bal1k", cameras=120, points=12000, seed=41)


@pytest.fixture(scope="module")
def trained():
    net = fg.LearnedPreconditioner(seed=11)
    for seed in (21, 22, 23):
        data = synthetic.generate("bal1k", cameras=120, points=12000, seed=seed)
        net.collect(fg.BalProblem.from_data(data), fg.Schur(9 * data.num_cameras, 9, 3),
                    fg.OptimizeOptions(max_iterations=6), probes=8, seed=seed * 100, kind="products")
    train_idx = list(range(net.system_count()))
    before = net.mean_loss(train_idx)
    net.train(steps=300, learning_rate=1e-3)
    after = net.mean_loss(train_idx)
    return net, before, after, len(train_idx)


def test_training_reduces_the_loss_on_held_out_systems(trained):
    net, before, after, n = trained
    assert n >= 6 and after < before
    # held-out system: the trained network against its untrained (block-Jacobi) self
    d = _held_out()
    b, _ = _bal_backend(d)
    idx = net.capture(b, 1e-3, probes=8, seed=999, kind="products")
    trained_loss = net.evaluate(idx)[0]
    fresh = fg.LearnedPreconditioner(seed=11)
    j = fresh.import_system(**{k: v for k, v in net.export_system(idx).items() if k != "damping"})
    untrained_loss = fresh.evaluate(j)[0]
    print(f"held-out loss: block-Jacobi {untrained_loss:.4f} -> learned {trained_loss:.4f}")
    assert trained_loss < untrained_loss


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_learned_pcg_keeps_the_step_and_reports_the_comparison(trained, precision):
    net = trained[0]
    d = _held_out()
    ref, _ = _bal_backend(d, precision=precision)
    lam = 1e-3
    step_bj = ref.solve_damped(lam).delta
    its_bj = ref.diagnostics().iterations
    b, _ = _bal_backend(d, precision=precision, preconditioner="learned")
    b.attach_learned(net)
    step = b.solve_damped(lam).delta
    di = b.diagnostics()
    print(f"{precision}: PCG iterations block-Jacobi {its_bj}, learned {di.learned_iterations}")
    # FP32 solves are reproducible to an iteration or two (atomic reduction order)
    assert abs(di.block_jacobi_iterations - its_bj) <= (0 if precision == "f64" else 2)
    assert di.iterations == di.learned_iterations + di.block_jacobi_iterations
    if di.learned_fallback == "more_iterations":
        assert di.learned_iterations > di.block_jacobi_iterations and di.preconditioner_used == "retained_blocks"
    else:
        assert di.learned_iterations <= di.block_jacobi_iterations and di.preconditioner_used == "learned"
    tol = 1e-7 if precision == "f64" else 1e-5
    assert np.linalg.norm(step - step_bj) <= tol * np.linalg.norm(step_bj)
    # after the comparison: a single solve with whichever preconditioner won
    b.solve_damped(lam * 2)
    d2 = b.diagnostics()
    assert d2.block_jacobi_iterations == 0 or d2.learned_fallback == "failed"


def test_lm_with_learned_preconditioner_reaches_the_f64_cost(trained):
    net = trained[0]
    d = _held_out()
    opts = fg.OptimizeOptions(max_iterations=8)
    ref = fg.LevenbergMarquardt(fg.Schur(9 * d.num_cameras, 9, 3))
    r0 = ref.solve_batch_with_outcome(fg.BalProblem.from_data(d), opts).statistics.cost
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision="f32", preconditioner="learned")
    b.attach_learned(net)
    out = fg.LevenbergMarquardt(b).solve_batch_with_outcome(fg.BalProblem.from_data(d), opts)
    assert abs(out.statistics.cost - r0) <= 1e-6 * r0
    assert out.work.linear_solve.iterations > 0


def test_learned_preconditioner_rejects_unsupported_widths():
    net = fg.LearnedPreconditioner()
    b = fg.Schur(24, 12, 3, preconditioner="learned")
    with pytest.raises(fg.UnsupportedStructure):
        b.attach_learned(net)


def test_training_set_of_uneven_systems_and_the_reported_comparison():
    """A training set in the shape of the learned-preconditioner workload
    (reduced camera systems of LM runs on problems of uneven size, uneven
    tracks), trained on the device; on a held-out problem the first learned
    solve reports both iteration counts and both device times, and the policy
    keeps the network exactly when it needed no more iterations and no more
    time than block-Jacobi."""
    net = fg.LearnedPreconditioner(seed=5)
    sizes = net.collect_set(6, cameras=(120, 200), points_per_camera=100, seed=3)
    assert net.system_count() == 6 and len(sizes) >= 2
    assert all(120 <= c <= 200 and p == 100 * c for c, p, _ in sizes)
    assert len({o / c for c, _, o in sizes}) > 1  # uneven observation counts per camera
    before = net.mean_loss()
    net.train(steps=200, learning_rate=1e-3)
    assert net.mean_loss() < before
    d = synthetic.generate("bal10k", cameras=160, points=16000, seed=77)
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision="f32", preconditioner="learned", coarse_correction=True)
    p = fg.BalProblem.from_data(d)
    b.prepare(p.dimension())
    p.linearize(b)
    b.prepare_damping(1e-6)
    b.attach_learned(net)
    b.solve_damped(1e-3)
    di = b.diagnostics()
    assert di.learned_iterations > 0 and di.block_jacobi_iterations > 0
    assert di.learned_seconds > 0 and di.block_jacobi_seconds > 0
    keep = di.learned_iterations <= di.block_jacobi_iterations and di.learned_seconds <= di.block_jacobi_seconds
    assert di.preconditioner_used == ("learned" if keep else "retained_blocks")
