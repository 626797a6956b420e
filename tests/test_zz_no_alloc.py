"""The allocation-free FP64 entry point, xk_diffraction_f64_noalloc.

It exists for callers that cannot let a library allocate device memory (their
device memory belongs to their own pool allocator, or their loop cannot pay
for cudaMalloc's implicit synchronisation). It must give what the allocating
FP64 entry point gives, call after call, although every call reuses the same
fixed scratch array inside the library.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import _lib, synth

pytestmark = pytest.mark.gpu

F64_TOL = 1e-10  # the FP64 path's parity tolerance used throughout the tests


def _device_arrays(torch, arrays):
    return [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda() for a in arrays]


def _dp(t):
    return ctypes.cast(ctypes.c_void_p(int(t.data_ptr())), ctypes.POINTER(ctypes.c_double))


def _noalloc(torch, d_rays, d_pix, n, m):
    lib = _lib.load()
    d_out = [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in range(4)]
    xr = _lib.XkRays(*[_dp(t) for t in d_rays])
    xp = _lib.XkPixels(*[_dp(t) for t in d_pix])
    xf = _lib.XkField(*[_dp(t) for t in d_out])
    stream = torch.cuda.current_stream()
    rc = lib.xk_diffraction_f64_noalloc(ctypes.byref(xr), n, ctypes.byref(xp), m,
                                        ctypes.byref(xf), ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc, [t.cpu().numpy() for t in d_out]


def _allocating(torch, ctx, d_rays, d_pix, m):
    d_out = [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in range(4)]
    xrt_rs.diffraction_integral_device(d_rays, d_pix, d_out, path="f64", ctx=ctx)
    return [t.cpu().numpy() for t in d_out]


def test_noalloc_matches_allocating_path_on_two_calls_in_a_row(ctx):
    torch = pytest.importorskip("torch")
    inputs = [synth.config0(seed=5), cases.random_case(3000, 700, seed=9, general_normals=True)]
    for rays, pix in inputs:
        rl, pl = cases.as_lists(rays, pix)
        d_rays = _device_arrays(torch, rl)
        d_pix = _device_arrays(torch, pl)
        n, m = len(rl[0]), len(pl[0])
        ref = _allocating(torch, ctx, d_rays, d_pix, m)
        rc, got = _noalloc(torch, d_rays, d_pix, n, m)
        assert rc == _lib.XK_OK
        assert cases.rel_l2(got, ref) <= F64_TOL


def test_noalloc_rejects_more_rays_than_its_scratch_holds(ctx):
    torch = pytest.importorskip("torch")
    n = 131072 + 1
    rays, pix = cases.random_case(n, 4, seed=1)
    rl, pl = cases.as_lists(rays, pix)
    rc, out = _noalloc(torch, _device_arrays(torch, rl), _device_arrays(torch, pl), n, 4)
    assert rc == _lib.XK_ERR_BUDGET
    assert all(np.all(o == 0) for o in out)  # nothing was launched


@pytest.mark.parametrize("n_rays,grid,line", [
    (2000, 256, 0),      # 2^16 screen points: the fixed area holds 8 ray ranges, the allocating path uses 19
    (64, 0, 600_000),    # more than 2^19 screen points: no room for partials, one ray range
])
def test_noalloc_where_its_scratch_caps_the_ray_split(ctx, oracle, n_rays, grid, line):
    """The two branches this entry point has of its own: fewer ray ranges than
    the allocating path (Kahan sums in another order) and a single range.
    Both agree with the allocating FP64 path and with the CPU oracle."""
    torch = pytest.importorskip("torch")
    rays, _ = cases.random_case(n_rays, 1, seed=31)
    if grid:
        pix = synth.grid_screen(grid, grid, 0.3, 1000.0)
    else:
        pix = synth.line_screen(line, 0.3, 1000.0)
    rl, pl = cases.as_lists(rays, pix)
    d_rays = _device_arrays(torch, rl)
    d_pix = _device_arrays(torch, pl)
    n, m = len(rl[0]), len(pl[0])
    ref = _allocating(torch, ctx, d_rays, d_pix, m)
    for _ in range(2):
        rc, got = _noalloc(torch, d_rays, d_pix, n, m)
        assert rc == _lib.XK_OK
        assert cases.rel_l2(got, ref) <= F64_TOL
    cpu = oracle.kahan_f64(rl, pl)
    assert cases.rel_l2(got, cpu) <= F64_TOL
