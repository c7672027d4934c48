"""mfista_nufft_forward_noalloc (the NUFFT forward operator that allocates no
GPU memory) against mfista_nufft_forward, through the C ABI.

The caller owns every buffer (here torch tensors on cuda:0) and passes
device pointers and a stream.  Two calls in a row on different grids and
point sets share the library's fixed scratch array; each must match the
allocating entry point within the FP64 operator tolerance used throughout
(1e-12 relative L2).  The file sorts last so that a run stopping at the
first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _noalloc(si):
    f = si.lib().mfista_nufft_forward_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    return f


def _case_128():
    from sparseimaging_b200 import synth
    rng = np.random.default_rng(128)
    u, v = synth.earth_rotation_uv(9, 60, seed=None, rng=rng)
    u_dx, v_dy = synth.scale_uv_to_radians(u, v, 128, synth.safe_kmax(128))
    return u_dx, v_dy, rng.random(128 * 128)


def test_noalloc_forward_matches_allocating_entry_point(gpulib, c0):
    import torch
    f = _noalloc(gpulib)
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(device=dev)
    u2, v2, x2 = _case_128()
    cases = [(c0["u"], c0["v"], 64, 64, c0["sky"]), (u2, v2, 128, 128, x2)]
    outs = []
    for u, v, nx, ny, x in cases:   # two calls in a row on the shared scratch
        du = torch.from_numpy(np.ascontiguousarray(u, np.float64)).to(dev)
        dv = torch.from_numpy(np.ascontiguousarray(v, np.float64)).to(dev)
        dx = torch.from_numpy(np.ascontiguousarray(x, np.float64)).to(dev)
        o_r = torch.full((u.size,), float("nan"), dtype=torch.float64, device=dev)
        o_i = torch.full((u.size,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        st = f(du.data_ptr(), dv.data_ptr(), u.size, nx, ny, dx.data_ptr(), o_r.data_ptr(), o_i.data_ptr(),
               stream.cuda_stream)
        assert st == 0
        stream.synchronize()
        outs.append((o_r.cpu().numpy(), o_i.cpu().numpy()))
    for (u, v, nx, ny, x), (o_r, o_i) in zip(cases, outs):
        fr, fi = gpulib.nufft_forward(u, v, nx, ny, x)
        assert np.all(np.isfinite(o_r)) and np.all(np.isfinite(o_i))
        assert rel(o_r + 1j * o_i, fr + 1j * fi) < 1e-12
    # the first case against the reference's own forward output, too
    assert rel(outs[0][0] + 1j * outs[0][1], c0["fwd_r"] + 1j * c0["fwd_i"]) < 1e-12


def test_noalloc_forward_takes_no_device_memory(gpulib, c0):
    """Once a device has the scratch array, a call leaves the device's free
    memory unchanged (cudaMemGetInfo before and after)."""
    import torch
    f = _noalloc(gpulib)
    dev = torch.device("cuda:0")
    u2, v2, x2 = _case_128()
    bufs = [torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(dev) for a in (u2, v2, x2)]
    o_r = torch.zeros(u2.size, dtype=torch.float64, device=dev)
    o_i = torch.zeros(u2.size, dtype=torch.float64, device=dev)
    args = (bufs[0].data_ptr(), bufs[1].data_ptr(), u2.size, 128, 128, bufs[2].data_ptr(), o_r.data_ptr(),
            o_i.data_ptr(), None)
    assert f(*args) == 0  # the device has its array and kernels from here on
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    assert f(*args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    fr, fi = gpulib.nufft_forward(u2, v2, 128, 128, x2)
    assert rel(o_r.cpu().numpy() + 1j * o_i.cpu().numpy(), fr + 1j * fi) < 1e-12


def test_noalloc_forward_rejects_sizes_beyond_its_scratch(gpulib):
    import torch
    f = _noalloc(gpulib)
    dev = torch.device("cuda:0")
    m = 64
    d = torch.zeros(m, dtype=torch.float64, device=dev)
    x = torch.zeros(1024 * 1024, dtype=torch.float64, device=dev)
    o = torch.full((m,), 7.0, dtype=torch.float64, device=dev)
    # a 1024 x 1024 image needs ~42 MB of grid: more than the fixed array
    assert f(d.data_ptr(), d.data_ptr(), m, 1024, 1024, x.data_ptr(), o.data_ptr(), o.data_ptr(), None) == 2
    # too many points for the array on a small grid
    big = 200000
    db = torch.zeros(big, dtype=torch.float64, device=dev)
    ob = torch.zeros(big, dtype=torch.float64, device=dev)
    assert f(db.data_ptr(), db.data_ptr(), big, 64, 64, x.data_ptr(), ob.data_ptr(), ob.data_ptr(), None) == 2
    torch.cuda.synchronize()
    assert torch.all(o == 7.0)
