"""ctr_sart_views_noalloc: the SART view update for callers that cannot
allocate device memory while they reconstruct (a pool that has reserved the
GPU, a real-time loop that must not stall on cudaMalloc/cudaFree).  Its ray
records live in a fixed 8 MiB array inside the library, so its detector limit
is 1,048,576 pixels.  Called through the C ABI and compared with
ctr_sart_views, which allocates, on two calls in a row, for every storage
type and update flag and for the tetrahedron beam; and shown to allocate
nothing on a fresh geometry.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from scan_configs import SMALL, TBCT, ctr_desc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SCANS = dict(SMALL, **TBCT)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _call(lib, g, vol, sino, beta, v0, n, noalloc, flags=0, seed=0):
    import gpu_b200
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        st = lib.ctr_sart_views_noalloc(g.h, vol.data_ptr(), gpu_b200.dtype_code(vol), sino.data_ptr(),
                                        gpu_b200.dtype_code(sino), beta, flags, seed, v0, n, stream)
    else:
        st = lib.ctr_sart_views(g.h, vol.data_ptr(), gpu_b200.dtype_code(vol), sino.data_ptr(),
                                gpu_b200.dtype_code(sino), beta, flags, seed, v0, n, None, None, stream)
    assert st == 0, gpu_b200.last_error()


def _problem(name, dtype):
    import gpu_b200
    cfg = SCANS[name]
    g = gpu_b200.Geometry(ctr_desc(cfg))
    rng = np.random.default_rng(41)
    truth = torch.from_numpy(rng.uniform(0, 0.05, g.vol_shape).astype(np.float32)).cuda()
    sino = torch.zeros((cfg["nviews"],) + g.view_shape, device="cuda")
    g.forward(truth, sino)
    return cfg, g, sino.to(dtype)


CASES = [("cube16", "f32", "plain"), ("fine_even", "f32", "plain"), ("cube16", "f16", "plain"),
         ("cube16", "bf16", "plain"), ("cube16", "f16", "stochastic"), ("cube16", "bf16", "stochastic"),
         ("cube16", "f32", "reference_bp"), ("fine_even", "f16", "reference_bp"), ("tbct_one", "f32", "plain"),
         ("tbct_one", "f32", "reference_bp"), ("tbct_one", "bf16", "stochastic")]


@pytest.mark.parametrize("name,dtype,mode", CASES)
def test_noalloc_matches_allocating_entry_point(name, dtype, mode):
    import gpu_b200
    tdt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[dtype]
    flags = {"plain": 0, "stochastic": gpu_b200.SART_STOCHASTIC_ROUND,
             "reference_bp": gpu_b200.SART_REFERENCE_BP}[mode]
    lib = gpu_b200.load_library()
    cfg, g, sino = _problem(name, tdt)
    a = torch.zeros(g.vol_shape, device="cuda", dtype=tdt)
    b = torch.zeros_like(a)
    half = cfg["nviews"] // 2
    # two calls in a row on each entry point; equal after each
    for v0, n in ((0, half), (half, cfg["nviews"] - half)):
        _call(lib, g, a, sino, 0.8, v0, n, noalloc=False, flags=flags, seed=7)
        _call(lib, g, b, sino, 0.8, v0, n, noalloc=True, flags=flags, seed=7)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
    assert a.float().abs().sum() > 0


def test_noalloc_allocates_nothing():
    """On a fresh geometry (no ray workspace yet) two calls leave the device's
    free memory unchanged, while the allocating entry point's first call on
    another fresh geometry takes its 8 MiB of ray records."""
    import gpu_b200
    lib = gpu_b200.load_library()
    cfg = dict(SMALL["cube16"], nu=1024, nv=1024, nviews=4)   # 1,048,576 rays: the limit
    warm = gpu_b200.Geometry(ctr_desc(cfg))                   # loads the kernels and looks the array up
    vol = torch.zeros(warm.vol_shape, device="cuda")
    sino = torch.rand((cfg["nviews"],) + warm.view_shape, device="cuda")
    _call(lib, warm, vol.clone(), sino, 0.8, 0, 2, noalloc=True)
    g = gpu_b200.Geometry(ctr_desc(cfg))
    a = vol.clone()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _call(lib, g, a, sino, 0.8, 0, 2, noalloc=True)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    _call(lib, g, a, sino, 0.8, 2, 2, noalloc=True)
    torch.cuda.synchronize()
    free2 = torch.cuda.mem_get_info()[0]
    assert free0 == free1 == free2
    g2 = gpu_b200.Geometry(ctr_desc(cfg))
    b = vol.clone()
    torch.cuda.synchronize()
    free3 = torch.cuda.mem_get_info()[0]
    _call(lib, g2, b, sino, 0.8, 0, 2, noalloc=False)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] <= free3 - (8 << 20)   # the measurement sees an allocation
    _call(lib, g2, b, sino, 0.8, 2, 2, noalloc=False)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


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


def test_noalloc_rejects_tiled_flag():
    import gpu_b200
    lib = gpu_b200.load_library()
    _, g, sino = _problem("cube16", torch.float32)
    vol = torch.zeros(g.vol_shape, device="cuda")
    st = lib.ctr_sart_views_noalloc(g.h, vol.data_ptr(), 0, sino.data_ptr(), 0, C.c_float(0.8),
                                    gpu_b200.SART_TILED, 0, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert st == 1
    assert "CTR_SART_TILED" in gpu_b200.last_error()
