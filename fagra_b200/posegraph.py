"""Deterministic synthetic SE(3) pose-graph windows (the batched-window workload).

A batch holds independent windows of uneven size. Window w has n_w poses
(uniform in [min_poses, max_poses]); its factors are, in emission order,
  - an anchor PosePrior on pose 0 (measurement = the true pose 0),
  - relative-pose factors i -> i+1 (odometry) for every consecutive pair,
  - round(loop_fraction * n_w) loop closures between distinct random pairs
    (i, j) with j >= i + 2, no pair repeated.
Relative measurements are z_ij = (x_i^-1 x_j) Exp([nt; nr]) with translation
noise nt ~ N(0, 0.05^2) and rotation noise nr ~ N(0, 0.01^2) per component.
True trajectories move about 1 m per step along the body x axis with small
random turns; initial estimates are the dead-reckoned odometry chain from the
true pose 0.

Poses are 7 doubles [qw, qx, qy, qz, tx, ty, tz]; tangents are body-frame
[v, w] with right increments (x (+) d = x Exp(d)), as in fagra's
examples/slam/geometry.rs. All randomness is the counter-based generator of
`synthetic` (seed, stream, index), so every window is reproducible alone.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .synthetic import normal, uniform


def _qmul(a, b):
    w = a[..., 0] * b[..., 0] - a[..., 1] * b[..., 1] - a[..., 2] * b[..., 2] - a[..., 3] * b[..., 3]
    x = a[..., 0] * b[..., 1] + a[..., 1] * b[..., 0] + a[..., 2] * b[..., 3] - a[..., 3] * b[..., 2]
    y = a[..., 0] * b[..., 2] - a[..., 1] * b[..., 3] + a[..., 2] * b[..., 0] + a[..., 3] * b[..., 1]
    z = a[..., 0] * b[..., 3] + a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1] + a[..., 3] * b[..., 0]
    return np.stack([w, x, y, z], axis=-1)


def _qrot(q, v):
    u = q[..., 1:]
    t = 2.0 * np.cross(u, v)
    return v + q[..., :1] * t + np.cross(u, t)


def compose(a, b):
    """SE(3) composition of (..., 7) poses."""
    q = _qmul(a[..., :4], b[..., :4])
    t = _qrot(a[..., :4], b[..., 4:]) + a[..., 4:]
    return np.concatenate([q, t], axis=-1)


def inverse(a):
    qi = a[..., :4] * np.array([1.0, -1.0, -1.0, -1.0])
    return np.concatenate([qi, -_qrot(qi, a[..., 4:])], axis=-1)


def exp(d):
    """SE(3) exponential of (..., 6) tangents [v, w] (closed form)."""
    v, w = d[..., :3], d[..., 3:]
    t2 = np.sum(w * w, axis=-1, keepdims=True)
    th = np.sqrt(t2)
    small = t2 < 1e-8
    ths = np.where(small, 1.0, th)
    a = np.where(small, 0.5 - t2 / 48.0, np.sin(0.5 * th) / ths)
    qw = np.cos(0.5 * th)
    b = np.where(small, 0.5 - t2 / 24.0, (1.0 - np.cos(th)) / np.where(small, 1.0, t2))
    c = np.where(small, 1.0 / 6.0 - t2 / 120.0, (th - np.sin(th)) / np.where(small, 1.0, t2 * ths))
    q = np.concatenate([qw, w * a], axis=-1)
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    wxv = np.cross(w, v)
    t = v + b * wxv + c * np.cross(w, wxv)
    return np.concatenate([q, t], axis=-1)


@dataclass
class WindowBatch:
    sizes: np.ndarray        # (W,) poses per window
    pose_offset: np.ndarray  # (W+1,)
    poses: np.ndarray        # (sum n, 7) initial estimates
    truth: np.ndarray        # (sum n, 7)
    prior: np.ndarray        # (W, 7) anchor measurement on each window's pose 0
    rel_offset: np.ndarray   # (W+1,)
    rel_ij: np.ndarray       # (R, 2) uint32, window-local pose indices
    rel_z: np.ndarray        # (R, 7)

    @property
    def windows(self) -> int:
        return len(self.sizes)

    def window(self, w: int):
        p0, p1 = self.pose_offset[w], self.pose_offset[w + 1]
        r0, r1 = self.rel_offset[w], self.rel_offset[w + 1]
        return (self.poses[p0:p1].copy(), self.prior[w].copy(), self.rel_ij[r0:r1].copy(),
                self.rel_z[r0:r1].copy())

    def dimension(self, w: int) -> int:
        return 6 * int(self.sizes[w])


def _loop_pairs(seed: int, w: int, n: int, loop_fraction: float):
    base = 1000 + 16 * w
    nl = int(round(loop_fraction * n))
    pairs = []
    seen = set()
    draws = uniform(seed, base + 2, 8 * max(nl, 1) + 16)
    pos = 0
    while len(pairs) < nl and pos + 1 < len(draws) and n >= 3:
        i = int(draws[pos] * n)
        j = int(draws[pos + 1] * n)
        pos += 2
        i, j = min(i, j), max(i, j)
        if j - i >= 2 and (i, j) not in seen:
            seen.add((i, j))
            pairs.append((i, j))
    return pairs


def generate(windows: int = 4096, *, min_poses: int = 20, max_poses: int = 300, loop_fraction: float = 0.1,
             seed: int = 5) -> WindowBatch:
    sizes = (min_poses + np.floor(uniform(seed, 900, windows) * (max_poses - min_poses + 1))).astype(np.int64)
    W, nmax = windows, int(sizes.max()) if windows else 0
    scale = np.array([0.1, 0.1, 0.05, 0.02, 0.02, 0.1])
    steps = np.zeros((W, nmax, 6))
    start = np.zeros((W, 6))
    ijs, noises = [], []
    for w in range(W):
        n = int(sizes[w])
        base = 1000 + 16 * w
        steps[w, :n] = normal(seed, base + 0, 6 * n).reshape(n, 6) * scale
        steps[w, :n, 0] += 1.0
        start[w] = normal(seed, base + 1, 6).reshape(6) * np.array([2.0, 2.0, 0.5, 0.1, 0.1, 1.0])
        ij = np.array([(k, k + 1) for k in range(n - 1)] + _loop_pairs(seed, w, n, loop_fraction),
                      dtype=np.uint32).reshape(-1, 2)
        ijs.append(ij)
        noises.append(normal(seed, base + 3, 6 * len(ij)).reshape(-1, 6) * np.array([0.05] * 3 + [0.01] * 3))
    # True trajectories, all windows at once (entries past a window's end are unused).
    truth = np.zeros((W, nmax, 7))
    truth[:, 0] = exp(start)
    step_exp = exp(steps)
    for k in range(1, nmax):
        truth[:, k] = compose(truth[:, k - 1], step_exp[:, k])
    pose_offset = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    rel_offset = np.concatenate([[0], np.cumsum([len(x) for x in ijs])]).astype(np.int64)
    flat_truth = np.concatenate([truth[w, :sizes[w]] for w in range(W)]) if W else np.zeros((0, 7))
    rel_ij = np.concatenate(ijs).astype(np.uint32) if W else np.zeros((0, 2), np.uint32)
    owner = np.repeat(np.arange(W), np.diff(rel_offset))
    gi = pose_offset[owner] + rel_ij[:, 0]
    gj = pose_offset[owner] + rel_ij[:, 1]
    rel = compose(inverse(flat_truth[gi]), flat_truth[gj])
    z = compose(rel, exp(np.concatenate(noises))) if W else np.zeros((0, 7))
    # Dead-reckoned initial estimates: factor k of a window is odometry k -> k+1.
    odo = np.zeros((W, max(nmax - 1, 0), 7))
    odo[..., 0] = 1.0
    for w in range(W):
        n = int(sizes[w])
        odo[w, :n - 1] = z[rel_offset[w]:rel_offset[w] + n - 1]
    init = np.zeros((W, nmax, 7))
    init[:, 0] = truth[:, 0]
    for k in range(1, nmax):
        init[:, k] = compose(init[:, k - 1], odo[:, k - 1])
    flat_init = np.concatenate([init[w, :sizes[w]] for w in range(W)]) if W else np.zeros((0, 7))
    return WindowBatch(sizes, pose_offset, flat_init, flat_truth, truth[:, 0].copy(), rel_offset, rel_ij, z)


# ---------------------------------------------------------------- device solver
WINDOW_OPTIONS = dict(max_iterations=20, gradient_tolerance=1e-6, step_tolerance=1e-10, cost_tolerance=1e-12)


class WindowSolver:
    """All windows of a batch on the device: LM over an all-retained DenseSchur
    per window, then square-root elimination of its oldest `removed` poses
    (fg_windows_* in libfagra_b200.so)."""

    def __init__(self, batch: WindowBatch, removed: int = 10, precision: str = "f64", device: int = 0):
        import ctypes as C
        from ._lib import lib
        from .errors import raise_for_status
        self._C, self._lib, self._raise = C, lib, raise_for_status
        self.batch = batch
        self.removed = removed
        po = np.ascontiguousarray(batch.pose_offset, np.uint64)
        ro = np.ascontiguousarray(batch.rel_offset, np.uint64)
        ij = np.ascontiguousarray(batch.rel_ij, np.uint32)
        h = C.c_void_p()
        u64 = C.POINTER(C.c_uint64)
        raise_for_status(lib.fg_windows_create(batch.windows, po.ctypes.data_as(u64), ro.ctypes.data_as(u64),
                                               ij.ctypes.data_as(C.POINTER(C.c_uint32)), removed,
                                               {"f64": 0, "f32": 1}[precision], device, C.byref(h)))
        self._h = h
        self._layout()

    def _layout(self):
        C, lib, h = self._C, self._lib, self._h
        u64 = C.POINTER(C.c_uint64)
        so = np.zeros(self.batch.windows + 1, np.uint64)
        ao = np.zeros(self.batch.windows + 1, np.uint64)
        self._raise(lib.fg_windows_prior_layout(h, so.ctypes.data_as(u64), ao.ctypes.data_as(u64), None))
        sep = np.zeros(max(int(so[-1]), 1), np.uint32)
        self._raise(lib.fg_windows_prior_layout(h, None, None, sep.ctypes.data_as(C.POINTER(C.c_uint32))))
        self.separator_offset, self.a_offset = so.astype(np.int64), ao.astype(np.int64)
        self.separators = sep[:int(so[-1])]

    def set_priors(self, priors):
        """Per window (A m x 6s, b m, refs s x 7): the prior r = b + sum_i A_i
        Log(ref_i^-1 x_i) on its first s poses in place of the anchor
        (Priors::update, src/marginalization.rs:157-231). The separator layout
        is re-read: prior poses past the removed ones join the separator."""
        C = self._C
        if len(priors) != self.batch.windows:
            raise ValueError("one prior per window")
        ps, pm, As, bs, rs = [], [], [], [], []
        for A, b, refs in priors:
            A = np.asarray(A, np.float64)
            refs = np.asarray(refs, np.float64).reshape(-1, 7)
            m, s6 = A.shape
            if s6 != 6 * len(refs):
                raise ValueError("A needs 6 columns per reference pose")
            ps.append(len(refs))
            pm.append(m)
            As.append(np.ascontiguousarray(A.T).reshape(-1))
            bs.append(np.asarray(b, np.float64).reshape(-1))
            rs.append(refs.reshape(-1))
        cat = lambda v: np.ascontiguousarray(np.concatenate(v) if v else np.zeros(1))
        psa, pma = np.asarray(ps, np.uint32), np.asarray(pm, np.uint32)
        A, b, r = cat(As), cat(bs), cat(rs)
        dp, u32 = C.POINTER(C.c_double), C.POINTER(C.c_uint32)
        self._raise(self._lib.fg_windows_set_priors(self._h, psa.ctypes.data_as(u32), pma.ctypes.data_as(u32),
                                                    A.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                                    r.ctypes.data_as(dp)))
        self._layout()

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fg_windows_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _opts(self, options, lm):
        from . import _lib
        o = dict(WINDOW_OPTIONS, **(options or {}))
        oc = _lib.OptimizeOptionsC(o["max_iterations"], o["gradient_tolerance"], o["step_tolerance"],
                                   o["cost_tolerance"])
        lc = _lib.LmOptionsC(*(lm or (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)))
        return oc, lc

    def upload(self, poses=None):
        C = self._C
        dp = C.POINTER(C.c_double)
        b = self.batch
        x = np.ascontiguousarray(b.poses if poses is None else poses, np.float64)
        pr = np.ascontiguousarray(b.prior, np.float64)
        z = np.ascontiguousarray(b.rel_z, np.float64)
        self._raise(self._lib.fg_windows_upload(self._h, x.ctypes.data_as(dp), pr.ctypes.data_as(dp),
                                                z.ctypes.data_as(dp)))

    def run(self, options=None, lm=None):
        oc, lc = self._opts(options, lm)
        C = self._C
        self._raise(self._lib.fg_windows_run(self._h, C.byref(oc), C.byref(lc)))

    def download(self):
        from . import _lib
        C = self._C
        dp = C.POINTER(C.c_double)
        b = self.batch
        poses = np.zeros_like(b.poses)
        reps = (_lib.WindowReportC * max(b.windows, 1))()
        a = np.zeros(max(int(self.a_offset[-1]), 1))
        bb = np.zeros(max(6 * int(self.separator_offset[-1]), 1))
        self._raise(self._lib.fg_windows_download(self._h, poses.ctypes.data_as(dp), reps, a.ctypes.data_as(dp),
                                                  bb.ctypes.data_as(dp)))
        return poses, list(reps)[:b.windows], a, bb

    def solve(self, options=None, lm=None):
        self.upload()
        self.run(options, lm)
        return self.download()

    def prior(self, w, report, a, b):
        """(A, b, constant, separator poses) of window w from downloaded buffers."""
        rows = int(report.prior_rows)
        s0, s1 = int(self.separator_offset[w]), int(self.separator_offset[w + 1])
        cols = 6 * (s1 - s0)
        A = a[int(self.a_offset[w]):int(self.a_offset[w]) + rows * cols].reshape(cols, rows).T.copy()
        return A, b[6 * s0:6 * s0 + rows].copy(), report.prior_constant

    def slide(self, poses, reports, a, b):
        """The next batch of a sliding window after this solve (slide_windows
        over this solve's poses, separators and priors)."""
        seps, pri = [], []
        for w in range(self.batch.windows):
            s0, s1 = int(self.separator_offset[w]), int(self.separator_offset[w + 1])
            seps.append([int(k) for k in self.separators[s0:s1]])
            A, bv, _ = self.prior(w, reports[w], a, b)
            pri.append((A, bv))
        return slide_windows(self.batch, self.removed, poses, seps, pri)

    def tuning(self):
        C = self._C
        panel, per = C.c_int(), C.c_int()
        ms = np.zeros(4)
        self._lib.fg_windows_tuning(self._h, C.byref(panel), C.byref(per), ms.ctypes.data_as(C.POINTER(C.c_double)))
        return panel.value, per.value, ms

    def stream(self):
        C = self._C
        s = C.c_void_p()
        self._lib.fg_windows_stream(self._h, C.byref(s))
        return s.value or 0


def slide_windows(batch: WindowBatch, removed: int, poses, separators, eliminations):
    """The next batch of a sliding window: window w keeps its poses past the
    `removed` oldest, separator poses first (in increasing order) then the
    rest, with the relative factors among them re-indexed; initial estimates
    are `poses` (the solve's result, all windows stacked); its prior is the
    elimination (A, b) on the separator poses linearized at those poses — the
    marginal prior of Priors::update (src/marginalization.rs:157-231).
    Returns (WindowBatch, priors) for WindowSolver.set_priors."""
    sizes, pose_rows, ij_rows, z_rows, priors, prior_x = [], [], [], [], [], []
    rel_off = [0]
    for w in range(batch.windows):
        p0, p1 = int(batch.pose_offset[w]), int(batch.pose_offset[w + 1])
        n = p1 - p0
        rm = min(removed, n)
        sep = list(separators[w])
        if not sep:
            raise ValueError("window %d keeps no separator pose" % w)
        keep = set(sep)
        order = sep + [k for k in range(rm, n) if k not in keep]
        local = {k: i for i, k in enumerate(order)}
        for f in range(int(batch.rel_offset[w]), int(batch.rel_offset[w + 1])):
            i, j = (int(v) for v in batch.rel_ij[f])
            if i >= rm and j >= rm:
                ij_rows.append((local[i], local[j]))
                z_rows.append(batch.rel_z[f])
        rel_off.append(len(ij_rows))
        x = np.asarray(poses[p0:p1], np.float64)[order]
        sizes.append(len(order))
        pose_rows.append(x)
        A, bv = eliminations[w]
        priors.append((np.asarray(A, np.float64), np.asarray(bv, np.float64), x[:len(sep)].copy()))
        prior_x.append(x[0])
    sizes = np.asarray(sizes, np.int64)
    out = WindowBatch(sizes, np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64), np.concatenate(pose_rows),
                      np.concatenate(pose_rows), np.asarray(prior_x, np.float64), np.asarray(rel_off, np.int64),
                      np.asarray(ij_rows, np.uint32).reshape(-1, 2), np.asarray(z_rows, np.float64).reshape(-1, 7))
    return out, priors
