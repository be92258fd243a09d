"""Device batches of bipartite emissions (fg_schur_accumulate_pairs_device):
the generic batched emission path for factor families other than BAL. The
same emissions passed one by one through fg_backend_accumulate (the
reference's CheckedSink -> LinearizedModel -> Schur::accumulate path,
src/optimization.rs:541-612, src/linear_model.rs:180-210, src/schur.rs:438-482)
give bit-identical index maps and values, the same steps, and the oracle's
steps; the CheckedSink errors are raised for the batch."""
import numpy as np
import pytest

import fagra_b200 as fg
import oracle

pytestmark = pytest.mark.gpu


def random_pairs(ncam, npt, cw, pw, rows, per_point=4, seed=0):
    rng = np.random.default_rng(seed)
    cams, pts = [], []
    for p in range(npt):
        for c in rng.choice(ncam, size=min(per_point, ncam), replace=False):
            cams.append(int(c))
            pts.append(p)
    order = rng.permutation(len(cams))  # an emission order that is neither camera- nor point-major
    cams, pts = np.array(cams, np.uint32)[order], np.array(pts, np.uint32)[order]
    n = len(cams)
    r = rng.normal(size=(n, rows))
    jr = rng.normal(size=(n, rows, cw))
    je = rng.normal(size=(n, rows, pw))
    return cams, pts, r, jr, je


def to_device_soa(torch, cams, pts, r, jr, je):
    dev = torch.device("cuda:0")
    n, rows, cw = jr.shape
    pw = je.shape[2]
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dt)  # noqa: E731
    return dict(cam=t(cams.astype(np.int32), torch.int32), pt=t(pts.astype(np.int32), torch.int32),
                r=t(r.T, torch.float64),                                           # r[i * n + k]
                jr=t(jr.transpose(2, 1, 0).reshape(cw * rows, n), torch.float64),  # [(j*rows+i)*n + k]
                je=t(je.transpose(2, 1, 0).reshape(pw * rows, n), torch.float64))


def host_emissions(ncam, cw, pw, cams, pts, r, jr, je):
    for k in range(len(cams)):
        yield r[k], [(int(cams[k]) * cw, jr[k]), (ncam * cw + int(pts[k]) * pw, je[k])]


def push_device(b, d, n, rows):
    b.accumulate_pairs_device(n, rows, d["cam"].data_ptr(), d["pt"].data_ptr(), d["r"].data_ptr(),
                              d["jr"].data_ptr(), d["je"].data_ptr())


@pytest.mark.parametrize("shape", [(6, 3, 4), (9, 3, 2), (5, 2, 3)])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_pair_batch_equals_host_emissions(shape, precision):
    import torch
    cw, pw, rows = shape
    ncam, npt = 40, 300
    cams, pts, r, jr, je = random_pairs(ncam, npt, cw, pw, rows, seed=cw * 10 + rows)
    dim = ncam * cw + npt * pw
    host = fg.Schur(ncam * cw, cw, pw, precision=precision)
    host.prepare(dim)
    for res, blocks in host_emissions(ncam, cw, pw, cams, pts, r, jr, je):
        host.accumulate(res, blocks)
    dev = fg.Schur(ncam * cw, cw, pw, precision=precision)
    dev.prepare(dim)
    d = to_device_soa(torch, cams, pts, r, jr, je)
    push_device(dev, d, len(cams), rows)
    assert dev.gradient_norm() == host.gradient_norm()
    for b in (host, dev):
        b.prepare_damping(1e-6)
    hs, ds = host.structure(), dev.structure()
    for key in ("blocks", "edges", "owners", "variables"):
        assert np.array_equal(hs[key], ds[key]), key
    hm, dm = host.model(), dev.model()
    for key in ("values", "negative_residual", "gradient", "scales", "gram"):
        assert np.array_equal(hm[key], dm[key]), key
    # the same device arithmetic on identical data; for the 9/3 shape the
    # single-pass operator's FP64 shared-memory atomics sum in whatever order
    # they arrive, so the steps agree to rounding rather than bit for bit
    for lam in (1e-3, 1.0):
        a, b = host.solve_damped(lam), dev.solve_damped(lam)
        assert np.linalg.norm(a.delta - b.delta) <= 1e-10 * np.linalg.norm(a.delta)
        assert abs(a.predicted_reduction - b.predicted_reduction) <= 1e-10 * abs(a.predicted_reduction)


def test_device_pair_batches_append_and_match_the_oracle():
    """Two batches with different row counts append in call order; the index
    maps equal the oracle's and the step equals its step (f64, 1e-9)."""
    import torch
    cw, pw, ncam, npt = 6, 3, 30, 200
    c1, p1, r1, j1, e1 = random_pairs(ncam, npt, cw, pw, 2, per_point=3, seed=1)
    c2, p2, r2, j2, e2 = random_pairs(ncam, npt, cw, pw, 4, per_point=2, seed=2)
    dim = ncam * cw + npt * pw
    dev = fg.Schur(ncam * cw, cw, pw)
    dev.prepare(dim)
    push_device(dev, to_device_soa(torch, c1, p1, r1, j1, e1), len(c1), 2)
    push_device(dev, to_device_soa(torch, c2, p2, r2, j2, e2), len(c2), 4)
    dev.gradient_norm()
    dev.prepare_damping(1e-6)
    o = oracle.Schur(ncam * cw, cw, pw)
    o.prepare(dim)
    for batch in ((c1, p1, r1, j1, e1), (c2, p2, r2, j2, e2)):
        for res, blocks in host_emissions(ncam, cw, pw, *batch):
            o.accumulate(res, blocks)
    o.prepare_damping(1e-6)
    ref = o.export()
    s = dev.structure()
    for key in ("blocks", "edges", "owners", "variables"):
        assert np.array_equal(s[key], ref[key]), key
    for lam in (1e-3, 0.5):
        _, delta, pred = o.solve_damped(lam)
        st = dev.solve_damped(lam)
        assert np.linalg.norm(st.delta - delta) <= 1e-9 * np.linalg.norm(delta)
        assert abs(st.predicted_reduction - pred) <= 1e-9 * abs(pred)


def test_device_pair_batch_errors():
    import torch
    cw, pw, ncam, npt = 6, 3, 10, 50
    cams, pts, r, jr, je = random_pairs(ncam, npt, cw, pw, 2, per_point=2, seed=3)
    dim = ncam * cw + npt * pw
    b = fg.Schur(ncam * cw, cw, pw)
    b.prepare(dim)
    bad = cams.copy()
    bad[7] = ncam  # a camera outside the layout
    with pytest.raises(fg.InvalidEmission):
        push_device(b, to_device_soa(torch, bad, pts, r, jr, je), len(cams), 2)
    nan = jr.copy()
    nan[3, 1, 2] = np.nan
    with pytest.raises(fg.InvalidEvaluation):
        push_device(b, to_device_soa(torch, cams, pts, r, nan, je), len(cams), 2)
    with pytest.raises(fg.DimensionMismatch):
        b.accumulate_pairs_device(len(cams), 17, 1, 1, 1, 1, 1)
    # the failing batches were dropped: a clean batch still solves
    push_device(b, to_device_soa(torch, cams, pts, r, jr, je), len(cams), 2)
    b.gradient_norm()
    b.prepare_damping(1e-6)
    assert np.all(np.isfinite(b.solve_damped(1e-2).delta))
