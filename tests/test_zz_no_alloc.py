"""ctr_sart_views_noalloc: the SART view update for callers that cannot
allocate device memory while they reconstruct (a pool that has reserved the
GPU, a real-time loop that must not stall on cudaMalloc/cudaFree).  Its ray
records live in a fixed 8 MiB array inside the library, so its detector limit
is 1,048,576 pixels.  Called through the C ABI and compared with
ctr_sart_views, which allocates, on two calls in a row.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from scan_configs import SMALL, ctr_desc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _call(lib, g, vol, sino, beta, v0, n, noalloc):
    import gpu_b200
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        st = lib.ctr_sart_views_noalloc(g.h, vol.data_ptr(), gpu_b200.dtype_code(vol), sino.data_ptr(),
                                        gpu_b200.dtype_code(sino), beta, 0, 0, v0, n, stream)
    else:
        st = lib.ctr_sart_views(g.h, vol.data_ptr(), gpu_b200.dtype_code(vol), sino.data_ptr(),
                                gpu_b200.dtype_code(sino), beta, 0, 0, v0, n, None, None, stream)
    assert st == 0, gpu_b200.last_error()


@pytest.mark.parametrize("name", ["cube16", "fine_even"])
def test_noalloc_matches_allocating_entry_point(name):
    import gpu_b200
    cfg = SMALL[name]
    lib = gpu_b200.load_library()
    g = gpu_b200.Geometry(ctr_desc(cfg))
    rng = np.random.default_rng(41)
    truth = torch.from_numpy(rng.uniform(0, 0.05, g.vol_shape).astype(np.float32)).cuda()
    sino = torch.zeros((cfg["nviews"],) + g.view_shape, device="cuda")
    g.forward(truth, sino)
    a = torch.zeros(g.vol_shape, device="cuda")
    b = torch.zeros_like(a)
    half = cfg["nviews"] // 2
    # two calls in a row on each entry point; equal after each
    for v0, n in ((0, half), (half, cfg["nviews"] - half)):
        _call(lib, g, a, sino, 0.8, v0, n, noalloc=False)
        _call(lib, g, b, sino, 0.8, v0, n, noalloc=True)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
    assert a.abs().sum() > 0


def test_noalloc_rejects_detector_beyond_limit():
    import gpu_b200
    cfg = dict(SMALL["cube16"], nu=2048, nv=1024)   # 2,097,152 pixels > 1,048,576
    lib = gpu_b200.load_library()
    g = gpu_b200.Geometry(ctr_desc(cfg))
    vol = torch.zeros(g.vol_shape, device="cuda")
    sino = torch.zeros((1,) + g.view_shape, device="cuda")
    st = lib.ctr_sart_views_noalloc(g.h, vol.data_ptr(), 0, sino.data_ptr(), 0, C.c_float(0.8), 0, 0, 0, 1,
                                    torch.cuda.current_stream().cuda_stream)
    assert st == 1
    assert "allocation-free limit" in gpu_b200.last_error()
