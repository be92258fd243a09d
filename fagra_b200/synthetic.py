"""Deterministic synthetic BAL-shaped bundle-adjustment problems.

Cameras use the BAL model of fagra's examples/bal/model.rs: 9 parameters
[angle-axis w (3), translation t (3), focal f, radial k1, k2], a point X
projects through p = R(w) X + t, q = -p.xy / p.z, pixel = f (1 + k1 r^2 +
k2 r^4) q; a point is in front of a camera when p.z < 0.

All randomness comes from a counter-based generator (SplitMix64 finalizer
over (seed, stream, index)) so every draw is reproducible on any machine and
independent of numpy's RNG implementation.

Named workloads:
  bal16   16 cameras on a circle of radius 5 around the origin, 1,000 points
          uniform in [-1,1]^3, 4 observing cameras per point.
  bal1k   1,000 cameras, 200,000 points, track length uniform in {3..8}.
  bal10k  10,000 cameras, 2,000,000 points, track length 2 + geometric (mean 4).
Intrinsics f = 500, k1, k2 ~ N(0, 1e-3); pixel noise N(0, 0.5); initial
estimates perturbed by N(0, 0.01) on rotation and translation and N(0, 0.05)
on point coordinates.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, n: int, offset: int = 0) -> np.ndarray:
    """n doubles in (0, 1) for (seed, stream), draws offset..offset+n-1."""
    with np.errstate(over="ignore"):
        key = _mix(np.array([np.uint64(seed) * GOLDEN + np.uint64(stream)], dtype=np.uint64))[0]
        idx = np.arange(offset, offset + n, dtype=np.uint64) + np.uint64(1)
        z = _mix(key + idx * GOLDEN)
    return ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (2.0 ** -53)


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normals (Box-Muller on consecutive uniform pairs)."""
    u = uniform(seed, stream, 2 * n).reshape(n, 2)
    return np.sqrt(-2.0 * np.log(u[:, 0])) * np.cos(2.0 * np.pi * u[:, 1])


def rotation_from_scaled_axis(w: np.ndarray) -> np.ndarray:
    """(n,3) angle-axis -> (n,3,3) rotations via the unit quaternion exp(w/2)."""
    v = w / 2.0
    nn = np.sum(v * v, axis=1)
    n = np.sqrt(nn)
    small = nn <= np.finfo(np.float64).eps ** 2
    s = np.where(small, 0.0, np.sin(n) / np.where(small, 1.0, n))
    qw = np.where(small, 1.0, np.cos(n))
    qi, qj, qk = v[:, 0] * s, v[:, 1] * s, v[:, 2] * s
    ww, ii, jj, kk = qw * qw, qi * qi, qj * qj, qk * qk
    ij, wk, wj, ik, jk, wi = 2 * qi * qj, 2 * qw * qk, 2 * qw * qj, 2 * qi * qk, 2 * qj * qk, 2 * qw * qi
    R = np.empty((len(w), 3, 3))
    R[:, 0, 0] = ww + ii - jj - kk; R[:, 0, 1] = ij - wk; R[:, 0, 2] = wj + ik
    R[:, 1, 0] = wk + ij; R[:, 1, 1] = ww - ii + jj - kk; R[:, 1, 2] = jk - wi
    R[:, 2, 0] = ik - wj; R[:, 2, 1] = wi + jk; R[:, 2, 2] = ww - ii - jj + kk
    return R


def rotation_log(R: np.ndarray) -> np.ndarray:
    """(n,3,3) rotations -> (n,3) angle-axis, robust at pi (Shepperd quaternion)."""
    n = len(R)
    q = np.zeros((n, 4))  # w, x, y, z
    tr = R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2]
    for i in range(n):
        m = R[i]
        cands = [tr[i], m[0, 0], m[1, 1], m[2, 2]]
        k = int(np.argmax(cands))
        if k == 0:
            s = np.sqrt(1.0 + tr[i]) * 2
            q[i] = [0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s]
        elif k == 1:
            s = np.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
            q[i] = [(m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s]
        elif k == 2:
            s = np.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
            q[i] = [(m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s]
        else:
            s = np.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
            q[i] = [(m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s]
    q[q[:, 0] < 0] *= -1
    v = q[:, 1:]
    nv = np.linalg.norm(v, axis=1)
    ang = 2.0 * np.arctan2(nv, q[:, 0])
    scale = np.where(nv > 0, ang / np.where(nv > 0, nv, 1.0), 2.0)
    return v * scale[:, None]


def project(cams: np.ndarray, pts: np.ndarray, oc: np.ndarray, op: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Pixels and camera-frame depth of every observation (vectorized BAL model)."""
    R = rotation_from_scaled_axis(cams[:, :3])
    X = pts[op]
    p = np.einsum("nij,nj->ni", R[oc], X) + cams[oc, 3:6]
    q = -p[:, :2] / p[:, 2:3]
    r2 = np.sum(q * q, axis=1)
    c = cams[oc]
    s = c[:, 6] * (1.0 + c[:, 7] * r2 + c[:, 8] * r2 * r2)
    return s[:, None] * q, p[:, 2]


@dataclass
class BalData:
    name: str
    cameras: np.ndarray       # (C, 9) initial estimates
    points: np.ndarray        # (P, 3) initial estimates
    obs_camera: np.ndarray    # (O,) uint32, insertion order
    obs_point: np.ndarray     # (O,) uint32
    obs_pixel: np.ndarray     # (O, 2)
    true_cameras: np.ndarray
    true_points: np.ndarray

    @property
    def num_cameras(self) -> int:
        return len(self.cameras)

    @property
    def num_points(self) -> int:
        return len(self.points)

    @property
    def num_observations(self) -> int:
        return len(self.obs_camera)

    def dimension(self) -> int:
        return 9 * self.num_cameras + 3 * self.num_points

    def emission_order(self) -> np.ndarray:
        """Observation indices in emission order: one Frame batch per camera,
        factors in insertion order within each frame (stable by camera)."""
        return np.argsort(self.obs_camera, kind="stable")


CONFIGS = {
    # name: (cameras, points, track rule, seed)
    "bal16": (16, 1000, ("fixed", 4), 1),
    "bal1k": (1000, 200_000, ("uniform", 3, 8), 2),
    "bal10k": (10_000, 2_000_000, ("geometric", 2, 1.0 / 3.0), 4),
}


def _track_lengths(rule, n: int, cams: int, seed: int) -> np.ndarray:
    if rule[0] == "fixed":
        k = np.full(n, rule[1], dtype=np.int64)
    elif rule[0] == "uniform":
        lo, hi = rule[1], rule[2]
        k = lo + np.floor(uniform(seed, 10, n) * (hi - lo + 1)).astype(np.int64)
    else:  # minimum + geometric number of failures with success probability p
        lo, p = rule[1], rule[2]
        g = np.floor(np.log(uniform(seed, 10, n)) / np.log1p(-p)).astype(np.int64)
        k = lo + g
    return np.minimum(k, min(cams, 64))


def _distinct_cameras(k: np.ndarray, cams: int, seed: int) -> np.ndarray:
    """For each point, k distinct cameras drawn uniformly; -1 pads unused slots."""
    n, K = len(k), int(k.max()) if len(k) else 0
    cand = np.floor(uniform(seed, 11, n * K).reshape(n, K) * cams).astype(np.int64)
    active = np.arange(K)[None, :] < k[:, None]
    rnd = 0
    while True:
        dup = np.zeros_like(active)
        for s in range(1, K):
            dup[:, s] = np.any(cand[:, :s] == cand[:, s:s + 1], axis=1)
        dup &= active
        cnt = int(dup.sum())
        if cnt == 0:
            break
        rnd += 1
        fresh = np.floor(uniform(seed, 100 + rnd, cnt) * cams).astype(np.int64)
        cand[dup] = fresh
    cand[~active] = -1
    return cand


def make_cameras(count: int, seed: int, radius: float = 5.0, focal: float = 500.0) -> np.ndarray:
    """Cameras on a circle in z = 0 looking at the origin (BAL convention)."""
    phi = 2.0 * np.pi * np.arange(count) / count
    centers = np.stack([radius * np.cos(phi), radius * np.sin(phi), np.zeros(count)], axis=1)
    z = centers / radius                      # origin lies at p.z = -radius
    y = np.tile(np.array([0.0, 0.0, 1.0]), (count, 1))
    x = np.cross(y, z)
    R = np.stack([x, y, z], axis=1)           # rows: camera axes in world frame
    w = rotation_log(R)
    Rw = rotation_from_scaled_axis(w)
    t = -np.einsum("nij,nj->ni", Rw, centers)
    k = normal(seed, 1, 2 * count).reshape(count, 2) * 1e-3
    cams = np.zeros((count, 9))
    cams[:, :3] = w
    cams[:, 3:6] = t
    cams[:, 6] = focal
    cams[:, 7:9] = k
    return cams


def generate(name: str = "bal16", *, cameras: int | None = None, points: int | None = None,
             seed: int | None = None) -> BalData:
    nc, npt, rule, s0 = CONFIGS[name]
    nc = cameras or nc
    npt = points or npt
    seed = s0 if seed is None else seed
    cams = make_cameras(nc, seed)
    pts = uniform(seed, 2, 3 * npt).reshape(npt, 3) * 2.0 - 1.0
    k = _track_lengths(rule, npt, nc, seed)
    sel = _distinct_cameras(k, nc, seed)
    rows, slots = np.nonzero(sel >= 0)        # point-major, slot order
    oc = sel[rows, slots].astype(np.uint32)
    op = rows.astype(np.uint32)
    pix, depth = project(cams, pts, oc, op)
    if not np.all(depth < 0):
        raise RuntimeError("generator produced an observation behind its camera")
    pix = pix + 0.5 * normal(seed, 3, 2 * len(oc)).reshape(-1, 2)
    init_c = cams.copy()
    init_c[:, :6] += 0.01 * normal(seed, 4, 6 * nc).reshape(nc, 6)
    init_p = pts + 0.05 * normal(seed, 5, 3 * npt).reshape(npt, 3)
    return BalData(name, init_c, init_p, oc, op, pix, cams, pts)


def parse_bal(text: str) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """BAL text format (examples/bal/model.rs:58-114): header, observations
    `camera point x y`, then 9 parameters per camera and 3 per point.
    Raises ValueError on truncated, invalid, nonfinite or trailing input."""
    tok = text.split()
    pos = 0

    def take(kind):
        nonlocal pos
        if pos >= len(tok):
            raise ValueError("truncated BAL input")
        t = tok[pos]
        pos += 1
        try:
            return kind(t)
        except ValueError:
            raise ValueError("invalid BAL token") from None

    nc, npt, no = take(int), take(int), take(int)
    if nc <= 0 or npt <= 0 or no <= 0:
        raise ValueError("empty BAL problem")
    oc = np.zeros(no, np.uint32)
    op = np.zeros(no, np.uint32)
    px = np.zeros((no, 2))
    for i in range(no):
        c, p = take(int), take(int)
        x, y = take(float), take(float)
        if c < 0 or c >= nc or p < 0 or p >= npt or not (np.isfinite(x) and np.isfinite(y)):
            raise ValueError("invalid observation index or value")
        oc[i], op[i], px[i] = c, p, (x, y)
    cams = np.array([take(float) for _ in range(9 * nc)]).reshape(nc, 9)
    pts = np.array([take(float) for _ in range(3 * npt)]).reshape(npt, 3)
    if not (np.all(np.isfinite(cams)) and np.all(np.isfinite(pts))):
        raise ValueError("nonfinite parameter")
    if pos != len(tok):
        raise ValueError("trailing BAL tokens")
    return cams, pts, oc, op, px
