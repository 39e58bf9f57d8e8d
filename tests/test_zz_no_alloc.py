"""The allocation-free MI entry point (regb_mi_cost_noalloc), for callers that cannot
allocate device memory at call time, must give the same costs as regb_mi_cost.

Runs last (file name) so a failure here cannot hide the rest of the suite; it works
both alone in a fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_mi_cost_twice():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tipl_b200 import _lib, build, phantom as ph
    import tipl_b200 as tb

    build.build()
    L = _lib.lib()
    rng = np.random.default_rng(ph.seed_for(2, 99))
    shape = (60, 70, 56)
    t, m, _ = ph.affine_pair(shape, rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    fdev = torch.from_numpy(f8).cuda()
    mdev = torch.from_numpy(m8).cuda()
    dims = np.array([shape[2], shape[1], shape[0]], np.int32)
    for call in range(2):
        Ts = np.array([tb.affine_to_matrix(ph.random_affine(rng, rot_deg=6, trans_vox=3), shape, (1, 1, 1), shape,
                                           (1, 1, 1)) for _ in range(12)], np.float32)
        ref = tb.mi_cost(f8, m8, Ts)
        out = torch.zeros(len(Ts), dtype=torch.float64, device="cuda")
        st = L.regb_mi_cost_noalloc(C.c_void_p(fdev.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                    C.c_void_p(mdev.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                    Ts.ctypes.data_as(C.c_void_p), len(Ts), C.c_void_p(out.data_ptr()), None)
        _lib.check(st)
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
    # more transforms than the static scratch holds: a clear error, nothing launched
    Ts = np.zeros((17, 12), np.float32)
    st = L.regb_mi_cost_noalloc(C.c_void_p(fdev.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                C.c_void_p(mdev.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                Ts.ctypes.data_as(C.c_void_p), 17, C.c_void_p(out.data_ptr()), None)
    assert st == _lib.REGB_ERR_ARG
    assert b"16" in L.regb_last_error()


def test_noalloc_refuses_stream_capture():
    """The call synchronises its stream, which a CUDA graph capture cannot hold: made while
    its stream is being captured, it returns REGB_ERR_ARG before any work and the capture
    ends normally."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tipl_b200 import _lib, build

    build.build()
    L = _lib.lib()
    dims = np.array([16, 16, 16], np.int32)
    vol = torch.zeros(16 * 16 * 16, dtype=torch.uint8, device="cuda")
    Ts = np.zeros((4, 12), np.float32)
    Ts[:, [0, 4, 8]] = 1.0
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        out.add_(1.0)
        st = L.regb_mi_cost_noalloc(C.c_void_p(vol.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                    C.c_void_p(vol.data_ptr()), dims.ctypes.data_as(C.c_void_p),
                                    Ts.ctypes.data_as(C.c_void_p), 4, C.c_void_p(out.data_ptr()),
                                    C.c_void_p(side.cuda_stream))
    assert st == _lib.REGB_ERR_ARG
    assert b"captured" in L.regb_last_error()
    g.replay()
    torch.cuda.synchronize()
    assert float(out[0]) == 1.0
