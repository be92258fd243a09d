"""fg_bal_cost_noalloc: the BAL objective for callers that cannot let the
library allocate device memory (their memory belongs to another allocator or to
a fixed budget). Inputs and the output are device buffers the caller owns; the
library's scratch is a fixed file-scope device array. Checked through the C ABI
against fg_bal_cost (which works through a problem handle that allocates), on
two calls in a row, since every call reuses the same scratch.

Kept in its own file, collected last, so a stop-at-first-failure run has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(torch, d):
    dev = torch.device("cuda:0")
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dt)  # noqa: E731
    return (t(d.cameras, torch.float64), t(d.points, torch.float64), t(d.obs_camera.astype(np.int32), torch.int32),
            t(d.obs_point.astype(np.int32), torch.int32), t(d.obs_pixel, torch.float64))


@pytest.mark.parametrize("name", ["bal16", "bal1k"])
def test_noalloc_cost_matches_handle_cost_on_two_calls(name):
    import torch
    import fagra_b200 as fg
    from fagra_b200 import _lib, synthetic
    from fagra_b200.errors import raise_for_status

    d = synthetic.generate(name)
    expected = fg.BalProblem.from_data(d).cost()
    cams, pts, oc, op, px = _device_inputs(torch, d)
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
    for _ in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        raise_for_status(_lib.lib.fg_bal_cost_noalloc(
            d.num_cameras, d.num_points, d.num_observations, C.c_void_p(cams.data_ptr()), C.c_void_p(pts.data_ptr()),
            C.c_void_p(oc.data_ptr()), C.c_void_p(op.data_ptr()), C.c_void_p(px.data_ptr()),
            C.c_void_p(out.data_ptr()), 0, None))
        torch.cuda.synchronize()
        cost, invalid = out.cpu().tolist()
        assert invalid == 0.0
        assert abs(cost - expected) <= 1e-12 * expected, (cost, expected)


def _call(d, cams, pts, oc, op, px, out):
    from fagra_b200 import _lib
    from fagra_b200.errors import raise_for_status
    raise_for_status(_lib.lib.fg_bal_cost_noalloc(
        d.num_cameras, d.num_points, d.num_observations, C.c_void_p(cams.data_ptr()), C.c_void_p(pts.data_ptr()),
        C.c_void_p(oc.data_ptr()), C.c_void_p(op.data_ptr()), C.c_void_p(px.data_ptr()),
        C.c_void_p(out.data_ptr()), 0, None))


def test_noalloc_cost_flags_out_of_range_indices_then_recovers():
    """An observation whose camera or point index is out of range is counted
    as an invalid evaluation on the device (out[1] = 1) and never read; the
    next call with valid indices reports a clean evaluation again, which also
    shows that the shared arrival counter was reset."""
    import torch
    import fagra_b200 as fg
    from fagra_b200 import synthetic

    d = synthetic.generate("bal16")
    expected = fg.BalProblem.from_data(d).cost()
    cams, pts, oc, op, px = _device_inputs(torch, d)
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda:0")
    bad_oc, bad_op = oc.clone(), op.clone()
    bad_oc[5] = d.num_cameras          # camera index one past the end
    bad_op[17] = d.num_points + 1000   # point index past the end
    for a, b in ((bad_oc, op), (oc, bad_op), (bad_oc, bad_op)):
        out.fill_(-1.0)
        _call(d, cams, pts, a, b, px, out)
        torch.cuda.synchronize()
        assert out[1].item() == 1.0
    out.fill_(-1.0)
    _call(d, cams, pts, oc, op, px, out)
    torch.cuda.synchronize()
    cost, invalid = out.cpu().tolist()
    assert invalid == 0.0
    assert abs(cost - expected) <= 1e-12 * expected


def test_noalloc_cost_leaves_device_memory_untouched():
    """After a warm-up call, a call changes the device's free memory by
    nothing: the entry point allocates no device memory of its own."""
    import torch
    from fagra_b200 import synthetic

    d = synthetic.generate("bal16")
    cams, pts, oc, op, px = _device_inputs(torch, d)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    _call(d, cams, pts, oc, op, px, out)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        _call(d, cams, pts, oc, op, px, out)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


def test_noalloc_cost_rejects_oversized_problems():
    import torch
    import fagra_b200 as fg
    from fagra_b200 import _lib
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = C.c_void_p(buf.data_ptr())
    code = _lib.lib.fg_bal_cost_noalloc(16385, 1, 1, p, p, p, p, p, p, 0, None)
    assert code == fg.InvalidOptions.code
    assert "16384" in fg.last_error()
