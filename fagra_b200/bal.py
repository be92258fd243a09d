"""Device-resident BAL problem: fagra's examples/bal/model.rs `Frame` batches
with `Reprojection` factors, evaluated and linearized by CUDA kernels."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import lib, dptr
from .errors import raise_for_status


class BalProblem:
    """Cameras (C,9), points (P,3) and observations (camera, point, pixel) in
    insertion order. One Frame batch per camera fixes the emission order."""

    def __init__(self, cameras, points, obs_camera, obs_point, obs_pixel, device: int = 0):
        cams = np.ascontiguousarray(np.asarray(cameras, np.float64).reshape(-1, 9))
        pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
        oc = np.ascontiguousarray(np.asarray(obs_camera, np.uint32))
        op = np.ascontiguousarray(np.asarray(obs_point, np.uint32))
        px = np.ascontiguousarray(np.asarray(obs_pixel, np.float64).reshape(-1, 2))
        h = C.c_void_p()
        u32 = C.POINTER(C.c_uint32)
        raise_for_status(lib.fg_bal_create(len(cams), len(pts), len(oc), cams.ctypes.data_as(dptr),
                                           pts.ctypes.data_as(dptr), oc.ctypes.data_as(u32),
                                           op.ctypes.data_as(u32), px.ctypes.data_as(dptr), device, C.byref(h)))
        self._bal_handle = h
        self.num_cameras, self.num_points, self.num_observations = len(cams), len(pts), len(oc)
        self.device = device

    @classmethod
    def from_data(cls, data, device: int = 0) -> "BalProblem":
        return cls(data.cameras, data.points, data.obs_camera, data.obs_point, data.obs_pixel, device)

    def dimension(self) -> int:
        return 9 * self.num_cameras + 3 * self.num_points

    def cost(self) -> float:
        out = C.c_double()
        raise_for_status(lib.fg_bal_cost(self._bal_handle, C.byref(out)))
        return out.value

    def parameters(self, out=None) -> tuple[np.ndarray, np.ndarray]:
        """Current cameras (C,9) and points (P,3); `out` = (cams, pts), C-contiguous
        float64 arrays of those shapes (e.g. pinned host memory), receives them."""
        if out is None:
            cams, pts = np.zeros((self.num_cameras, 9)), np.zeros((self.num_points, 3))
        else:
            cams, pts = out
            for a, n in ((cams, 9 * self.num_cameras), (pts, 3 * self.num_points)):
                if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != n:
                    raise ValueError("out arrays must be C-contiguous float64 of the parameter shapes")
        raise_for_status(lib.fg_bal_get_parameters(self._bal_handle, cams.ctypes.data_as(dptr),
                                                   pts.ctypes.data_as(dptr)))
        return cams, pts

    def set_parameters(self, cameras, points) -> None:
        cams = np.ascontiguousarray(np.asarray(cameras, np.float64))
        pts = np.ascontiguousarray(np.asarray(points, np.float64))
        raise_for_status(lib.fg_bal_set_parameters(self._bal_handle, cams.ctypes.data_as(dptr),
                                                   pts.ctypes.data_as(dptr)))

    def linearize(self, backend) -> None:
        """Workspace::linearize for these frames, straight into the backend."""
        raise_for_status(lib.fg_bal_linearize(self._bal_handle, backend.handle))

    def close(self) -> None:
        if getattr(self, "_bal_handle", None):
            lib.fg_bal_destroy(self._bal_handle)
            self._bal_handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
