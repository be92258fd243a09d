"""Learned block preconditioner for the Schur backend's reduced camera system
(C ABI `fg_gnn_*`; no fagra counterpart).

A message-passing network over the camera covisibility graph reshapes the
retained block-Jacobi preconditioner of fagra's Schur backend
(src/schur.rs:658-682): per camera it emits A_c = I + 0.1 tril(O_c) and the
preconditioner block L_c^-T (A_c A_c^T + 1e-3 I) L_c^-1, with L_c the
block-Jacobi factor, so the preconditioner is always SPD and an untrained
network is block-Jacobi. GEMMs run on the tensor cores with BF16 weights and
operands and FP32 accumulation; training (Adam) runs on the device over
reduced camera systems captured from the backend, typically on every accepted
LM step (`collect`).

    net = LearnedPreconditioner(seed=1)
    net.collect(problem, Schur(9 * C, 9, 3))      # LM run, one system per accepted step
    net.train(steps=400, learning_rate=1e-3)
    backend = Schur(9 * C, 9, 3, preconditioner="learned")
    backend.attach_learned(net)
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import lib
from .errors import raise_for_status

size_t = C.c_size_t
fptr = C.POINTER(C.c_float)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(fptr)


class LearnedPreconditioner:
    FEATURES = 64
    HIDDEN = 64

    def __init__(self, seed: int = 0, device: int = 0):
        h = C.c_void_p()
        raise_for_status(lib.fg_gnn_create(seed, device, C.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.fg_gnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters
    def parameter_count(self) -> int:
        n = size_t()
        raise_for_status(lib.fg_gnn_parameter_count(self._h, C.byref(n)))
        return n.value

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.parameter_count(), np.float32)
        raise_for_status(lib.fg_gnn_get_parameters(self._h, _fp(out)))
        return out

    def set_parameters(self, flat) -> None:
        a = np.ascontiguousarray(np.asarray(flat, np.float32))
        if a.size != self.parameter_count():
            raise ValueError("parameter vector has the wrong length")
        raise_for_status(lib.fg_gnn_set_parameters(self._h, _fp(a)))

    def save(self, path) -> None:
        np.save(path, self.parameters())

    def load(self, path) -> None:
        self.set_parameters(np.load(path))

    # ---- training systems
    PROBES = {"products": 0, "solves": 1}

    def capture(self, backend, damping: float, probes: int = 8, seed: int = 0, kind: str = "products") -> int:
        """The reduced camera system of a prepared Schur backend at `damping`.
        kind "products": Gaussian x, y = S_hat x; "solves": Gaussian y, x = S_hat^-1 y."""
        idx = size_t()
        raise_for_status(lib.fg_schur_capture_system(backend.handle, self._h, damping, probes, seed,
                                                     self.PROBES[kind], C.byref(idx)))
        return idx.value

    def collect(self, problem, backend, options=None, probes: int = 8, seed: int = 0, lm_options=None,
                kind: str = "products"):
        """Run LevenbergMarquardt on `problem` with `backend`, capturing the
        reduced camera system at every accepted step; returns the LmOutcome."""
        from .optimize import LevenbergMarquardt
        lm = LevenbergMarquardt(backend)
        if lm_options is not None:
            lm.options = lm_options
        count = [0]

        def on_accept(stats):
            self.capture(backend, max(stats.damping, 1e-12), probes, seed + count[0], kind)
            count[0] += 1

        lm.on_accept = on_accept
        return lm.solve_batch_with_outcome(problem, options)

    def collect_set(self, systems: int, *, cameras=(200, 2000), points_per_camera: int = 200, seed: int = 0,
                    max_lm_iterations: int = 4, probes: int = 8, kind: str = "products", device: int = 0):
        """A training set of `systems` reduced camera systems from LM runs on
        seeded BAL problems of uneven size: camera counts uniform in
        [cameras[0], cameras[1]], points_per_camera points per camera (the
        defaults span 200-2,000 cameras and 40,000-400,000 points), track
        lengths 2 + geometric with mean 4 (uneven observation counts per camera
        and point); one system per accepted LM step. Returns the (cameras,
        points, observations) of every problem used."""
        from .backend import Schur
        from .bal import BalProblem
        from .optimize import OptimizeOptions
        from .synthetic import generate, uniform
        goal = self.system_count() + systems
        sizes, k = [], 0
        while self.system_count() < goal:
            u = float(uniform(seed, 77, 1, offset=k)[0])
            nc = int(cameras[0] + u * (cameras[1] - cameras[0] + 1))
            d = generate("bal10k", cameras=nc, points=points_per_camera * nc, seed=seed * 7919 + 1000 + k)
            left = goal - self.system_count()
            self.collect(BalProblem.from_data(d, device=device), Schur(9 * nc, 9, 3, precision="f32", device=device),
                         OptimizeOptions(max_iterations=min(max_lm_iterations, left)), probes=probes,
                         seed=seed * 104729 + 31 * k, kind=kind)
            sizes.append((d.num_cameras, d.num_points, d.num_observations))
            k += 1
        return sizes

    def import_system(self, features, adjacency, probe_x, probe_y, mask) -> int:
        f = np.ascontiguousarray(features, np.float32)
        a = np.ascontiguousarray(adjacency, np.float32)
        x = np.ascontiguousarray(probe_x, np.float32)
        y = np.ascontiguousarray(probe_y, np.float32)
        m = np.ascontiguousarray(mask, np.uint8)
        K, Cn, w = x.shape
        idx = size_t()
        raise_for_status(lib.fg_gnn_import_system(self._h, Cn, w, K, _fp(f), _fp(a), _fp(x), _fp(y),
                                                  m.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(idx)))
        return idx.value

    def system_count(self) -> int:
        n = size_t()
        raise_for_status(lib.fg_gnn_system_count(self._h, C.byref(n)))
        return n.value

    def export_system(self, index: int) -> dict:
        c, w, k = size_t(), size_t(), size_t()
        raise_for_status(lib.fg_gnn_system_size(self._h, index, C.byref(c), C.byref(w), C.byref(k)))
        Cn, W, K = c.value, w.value, k.value
        out = dict(features=np.zeros((Cn, self.FEATURES), np.float32), adjacency=np.zeros((Cn, Cn), np.float32),
                   probe_x=np.zeros((K, Cn, W), np.float32), probe_y=np.zeros((K, Cn, W), np.float32),
                   mask=np.zeros(Cn, np.uint8))
        lam = C.c_double()
        raise_for_status(lib.fg_gnn_export_system(self._h, index, _fp(out["features"]), _fp(out["adjacency"]),
                                                  _fp(out["probe_x"]), _fp(out["probe_y"]),
                                                  out["mask"].ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(lam)))
        out["damping"] = lam.value
        return out

    def clear_systems(self) -> None:
        raise_for_status(lib.fg_gnn_clear_systems(self._h))

    # ---- training
    def evaluate(self, index: int, gradient: bool = False):
        """(loss, gradient or None, outputs C x 64) of one system."""
        c = size_t()
        raise_for_status(lib.fg_gnn_system_size(self._h, index, C.byref(c), None, None))
        loss = C.c_double()
        g = np.zeros(self.parameter_count(), np.float32) if gradient else None
        o = np.zeros((c.value, self.HIDDEN), np.float32)
        raise_for_status(lib.fg_gnn_evaluate(self._h, index, C.byref(loss), _fp(g) if gradient else None, _fp(o)))
        return loss.value, g, o

    def train(self, steps: int, learning_rate: float = 1e-3) -> float:
        """`steps` Adam steps over the captured systems; returns the mean loss."""
        out = C.c_double()
        raise_for_status(lib.fg_gnn_train(self._h, steps, learning_rate, C.byref(out)))
        return out.value

    def mean_loss(self, indices: Optional[list] = None) -> float:
        idx = range(self.system_count()) if indices is None else indices
        return float(np.mean([self.evaluate(i)[0] for i in idx]))
