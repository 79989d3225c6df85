"""Parity at the benchmark's full size: the 512^3 volume (0.5 mm), 1024x768
detector (0.4 mm), 1024 views, DSO 1000 mm, DOD -500 mm, the
tetrahedron-beam scan (512^3 x 0.1 mm, 64 sources x 16 x 1024), and the
large mixed-precision scan (1024^3 x 0.25 mm, 1024x1024 detector x 0.3 mm,
1024 views; its FP32 and FP16 projections).

The oracle projects and updates a few whole views of these scans in seconds
(OpenMP), so the checks are the small scans' checks on spread-out views:
ray sums and voxel index sequences bit-exact, a SART view update bit-exact
against the restated engine algorithm, and the dot product <Ax, y> =
<x, A^T y> to 1e-6 over several views."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SCAN = dict(nx=512, ny=512, nz=512, vx=0.5, nu=1024, nv=768, du=0.4, dso=1000.0, dod=-500.0, nviews=1024)
TBCT_SCAN = dict(nx=512, ny=512, nz=512, vx=0.1, nu=1024, nv=16, du=0.12, dso=200.0, dod=-200.0, nviews=360,
                 us_rate=1.0, ct_style=3, n_sources=64)
LARGE = dict(nx=1024, ny=1024, nz=1024, vx=0.25, nu=1024, nv=1024, du=0.3, dso=1000.0, dod=-500.0, nviews=1024)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def scan(cfg, oracle_mod):
    import gpu_b200
    us = cfg.get("us_rate", 360.0 / cfg["nviews"])
    g = gpu_b200.Geometry(gpu_b200.make_desc(cfg["nx"], cfg["ny"], cfg["nz"], cfg["vx"], cfg["nu"], cfg["nv"],
                                             cfg["du"], cfg["dso"], cfg["dod"], cfg["nviews"], us_rate=us,
                                             ct_style=cfg.get("ct_style", 0), n_sources=cfg.get("n_sources", 0)))
    o = oracle_mod.Oracle(oracle_mod.make_desc(cfg["nx"], cfg["ny"], cfg["nz"], cfg["nu"], cfg["nv"], cfg["nviews"],
                                               cfg["vx"], cfg["du"], cfg["dso"], cfg["dod"], us_rate=us,
                                               ct_style=cfg.get("ct_style", 0), n_sources=cfg.get("n_sources", 0)))
    assert o.view_shape == g.view_shape
    # seeded ellipsoids over the volume, voxelised on the device
    half = 0.5 * cfg["nx"] * cfg["vx"]
    p = oracle_mod.random_ellipsoids(np.random.default_rng(512), 12, 0.5 * half, (0.05 * half, 0.6 * half),
                                     (0.01 / cfg["vx"], 0.03 / cfg["vx"]))
    vol = torch.zeros(g.vol_shape, device="cuda")
    g.phantom_voxelize(p, vol)
    return g, o, vol


@pytest.mark.parametrize("cfg", [SCAN, TBCT_SCAN, LARGE], ids=["cone512", "tbct512", "cone1024"])
def test_forward_and_traversal_bit_exact(cfg, oracle_built):
    g, o, vol = scan(cfg, oracle_built)
    h = vol.cpu().numpy()
    views = [0, cfg["nviews"] // 3 + 1, cfg["nviews"] - 5][: 2 if cfg is LARGE else 3]
    nseg = torch.zeros(g.view_shape, dtype=torch.int32, device="cuda")
    hsh = torch.zeros(g.view_shape, dtype=torch.int64, device="cuda")
    ln = torch.zeros(g.view_shape, dtype=torch.float32, device="cuda")
    for j in views:
        out = torch.zeros((1,) + g.view_shape, device="cuda")
        g.forward(vol, out, j, 1)
        want = o.forward_view(h, j, 0)
        assert np.count_nonzero(want) > 0.1 * want.size
        np.testing.assert_array_equal(bits(out[0].cpu().numpy()), bits(want), err_msg=f"view {j}")
        g.forward_trace(vol, j, nseg, hsh, ln)
        n_ref, h_ref, l_ref = o.forward_trace(h, j)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(nseg.cpu().numpy(), n_ref)
        np.testing.assert_array_equal(hsh.cpu().numpy().view(np.uint64), h_ref)
        np.testing.assert_array_equal(bits(ln.cpu().numpy()), bits(l_ref))


@pytest.mark.parametrize("cfg", [SCAN, TBCT_SCAN], ids=["cone512", "tbct512"])
def test_sart_view_update_bit_exact(cfg, oracle_built):
    """One SART view (projector correction, then the gather update) on the
    full-size scan from a non-zero volume, against the restated engine
    algorithm (for the tetrahedron beam: its sources kept per voxel, bands
    summed in source order)."""
    g, o, vol = scan(cfg, oracle_built)
    h = vol.cpu().numpy()
    j = cfg["nviews"] // 2 + 5
    # measured data of a brighter object, placed at view j: a non-trivial correction
    b = torch.zeros((cfg["nviews"],) + g.view_shape, device="cuda")
    g.forward(vol * 1.05, b[j:j + 1], j, 1)
    bj = b[j].cpu().numpy()
    x = vol.clone()
    g.sart_views(x, b, 0.8, j, 1)
    corr = o.forward_view(h, j, 1, bj)
    want = o.backproject_gather(h, corr, j, 0.8)
    got = x.cpu().numpy()
    assert np.count_nonzero(got != h) > 0.05 * h.size
    np.testing.assert_array_equal(bits(got), bits(want))


@pytest.mark.parametrize("cfg", [SCAN, TBCT_SCAN, LARGE], ids=["cone512", "tbct512", "cone1024"])
def test_dot_product_full_size(cfg, oracle_built):
    """<Ax, y> = <x, A^T y> to 1e-6 relative over 8 views spread over the scan
    (x uniform over the voxels, y normal over the detector bins)."""
    g, _, _ = scan(cfg, oracle_built)
    gen = torch.Generator(device="cuda").manual_seed(8)
    x = torch.rand(g.vol_shape, device="cuda", generator=gen)
    for v0 in (0, cfg["nviews"] // 2 + 3):
        y = torch.randn((4,) + g.view_shape, device="cuda", generator=gen)
        a, b = g.dot_test(x, y, v0, 4)
        assert abs(a - b) <= 1e-6 * max(abs(a), abs(b)), (a, b)


@pytest.mark.parametrize("cfg", [SCAN, TBCT_SCAN], ids=["cone512", "tbct512"])
def test_sart_view_reference_backprojector_full_size(cfg, oracle_built):
    """CTR_SART_REFERENCE_BP at full size: one SART view from a non-zero volume
    equals the reference's backprojection arithmetic (the C restatement pinned
    to the reference's kernels) bit for bit."""
    import gpu_b200
    g, o, vol = scan(cfg, oracle_built)
    h = vol.cpu().numpy()
    j = (cfg["nviews"] // 2 + 189) % cfg["nviews"]
    b = torch.zeros((cfg["nviews"],) + g.view_shape, device="cuda")
    g.forward(vol * 1.05, b[j:j + 1], j, 1)
    x = vol.clone()
    g.sart_views(x, b, 0.8, j, 1, flags=gpu_b200.SART_REFERENCE_BP)
    corr = o.forward_view(h, j, 1, b[j].cpu().numpy())
    want = o.backproject_ref(h, corr, j, 0.8, 1)
    got = x.cpu().numpy()
    assert np.count_nonzero(got != h) > 0.05 * h.size
    np.testing.assert_array_equal(bits(got), bits(want))



def test_large_scan_half_precision_forward(oracle_built):
    """The 1024^3 scan stored in FP16 and BF16: each projection equals the
    oracle's FP32 projection of the widened volume, bit for bit (one view
    each; the storage is widened exactly, the arithmetic is the FP32 one)."""
    g, o, vol = scan(LARGE, oracle_built)
    for dt, j in ((torch.float16, 77), (torch.bfloat16, 611)):
        lo = vol.to(dt)
        del vol
        out = torch.zeros((1,) + g.view_shape, device="cuda")
        g.forward(lo, out, j, 1)
        want = o.forward_view(lo.float().cpu().numpy(), j, 0)
        assert np.count_nonzero(want) > 0.1 * want.size
        np.testing.assert_array_equal(bits(out[0].cpu().numpy()), bits(want), err_msg=str(dt))
        vol = lo.float()
        del lo
