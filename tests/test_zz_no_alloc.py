"""vg_max_wave_speed_noalloc: the allocation-free CFL maximum, checked against vg_max_wave_speed.

Callers that own all device memory through their own pool allocator cannot let a library call
cudaMalloc or cudaFree (a foreign allocation escapes their budget, and cudaFree synchronises the device under
their other streams).  The entry point takes a state the caller already holds on the device and keeps its
partial maxima in a fixed array inside the library image.  This file is collected last, so a run that stops
at the first failure has already run every other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from vanguard_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _noalloc(vg, torch, model, planes_np, params):
    """Call the entry point on a device copy of the reference-order planes; returns the device result."""
    dev = torch.from_numpy(np.ascontiguousarray(planes_np)).cuda()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    ny, nx = (planes_np.shape[1], planes_np.shape[2]) if planes_np.ndim == 3 else (1, planes_np.shape[1])
    stream = torch.cuda.current_stream().cuda_stream
    import ctypes
    vg.max_wave_speed_noalloc(model, dev.data_ptr(), nx * ny, nx, nx, ny, params, out.data_ptr(),
                              ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return float(out.item())


def _existing(vg, model, planes_np, params, boundary=0):
    ny, nx = (planes_np.shape[1], planes_np.shape[2]) if planes_np.ndim == 3 else (1, planes_np.shape[1])
    with vg.Solver(model, nx, ny, params, boundary=boundary) as s:
        s.upload(planes_np)
        return s.max_wave_speed()


CASES = [
    ("euler2d", 0, lambda: wl.euler_quadrants_2d(257, 129, seed=41), wl.euler_params(1.4)),
    ("euler2d_b", 0, lambda: wl.euler_quadrants_2d(300, 211, seed=42), wl.euler_params(1.4)),
    ("euler1d", 0, lambda: wl.sod_1d(1000, left=(1.0, 0.75, 1.0)), wl.euler_params(1.4)),
    ("mhd2d", 1, lambda: wl.mhd_vortex_2d(130, 96, seed=43), wl.mhd_params(5 / 3)),
]


@pytest.mark.parametrize("name,model,init,params", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_existing_entry_point_twice(gpu, name, model, init, params):
    import torch
    first = init()
    second = first.copy()
    second[0] *= 0.5  # a different state for the second call: lower density, faster sound speed
    for planes in (first, second):  # two calls in a row share the scratch array
        got = _noalloc(gpu, torch, model, planes, params)
        want = _existing(gpu, model, planes, params)
        assert got == want, (name, got, want)


def test_noalloc_rejects_rows_beyond_scratch(gpu):
    import torch
    dev = torch.zeros(6 * 4, dtype=torch.float64, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    rows = gpu.NOALLOC_MAX_ROWS + 1
    with pytest.raises(gpu.VgError) as e:
        gpu.max_wave_speed_noalloc(0, dev.data_ptr(), 4 * rows, 4, 4, rows, wl.euler_params(1.4), out.data_ptr())
    assert e.value.status == gpu.VG_EINVAL
    assert "VG_NOALLOC_MAX_ROWS" in str(e.value)


def test_noalloc_padded_strides(gpu):
    """Rows padded past nx and planes spaced past row_stride * ny, with the padding holding a state far faster than
    any cell: the padding must not be read, and the result must equal vg_max_wave_speed's, on two calls in a row."""
    import ctypes
    import torch
    W = wl.euler_quadrants_2d(100, 37, seed=44)
    nv, ny, nx = W.shape
    pitch, gap = 128, 96
    ps = ny * pitch + gap
    buf = torch.ones(nv * ps, dtype=torch.float64, device="cuda")
    buf[1 * ps:2 * ps] = 1e10          # u in the padding: a wave speed that would dominate if it were read
    for v in range(nv):
        buf[v * ps: v * ps + ny * pitch].view(ny, pitch)[:, :nx] = torch.from_numpy(W[v]).cuda()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    want = _existing(gpu, 0, W, wl.euler_params(1.4))
    for _ in range(2):
        out.fill_(-1.0)
        gpu.max_wave_speed_noalloc(0, buf.data_ptr(), ps, pitch, nx, ny, wl.euler_params(1.4), out.data_ptr(),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert float(out.item()) == want
