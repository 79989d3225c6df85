"""CTR_GEOM_FAST_SUMS: the projector accumulates (alpha step) x (voxel value)
with fused multiply-adds and applies the chord factor once per ray.  The
traversal is unchanged, so every ray visits the voxels of the reference's
sequence; only the rounding of the sums differs.  On volumes of independent
random values a ray that visited a different voxel would be off by about one
voxel's share of its sum (1e-3 and more), so agreement to 1e-5 relative with
the exact sums also shows the visited voxels are the same."""
import numpy as np
import pytest

from scan_configs import CONFIG0, SMALL, TBCT, ctr_desc, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SCANS = dict(SMALL, **TBCT, config0=CONFIG0)
REL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel_err(got, want):
    return float(np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-30)))


@pytest.mark.parametrize("name", ["cube16", "odd", "aniso", "tbct", "config0"])
def test_fast_sums_within_1e5_of_the_exact_sums(name, oracle_built):
    import gpu_b200
    cfg = SCANS[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    g = gpu_b200.Geometry(ctr_desc(cfg, fast_sums=True))
    rng = np.random.default_rng(5)
    vol = rng.uniform(0.01, 1.0, o.vol_shape).astype(np.float32)
    views = range(min(cfg["nviews"], 8))
    got = torch.zeros((len(views),) + o.view_shape, device="cuda")
    g.forward(torch.from_numpy(vol).cuda(), got, 0, len(views))
    want = np.stack([o.forward_view(vol, j, 0) for j in views])
    hit = want > 0
    assert np.array_equal(got.cpu().numpy() > 0, hit)           # the same rays pass the zero-length rule
    err = rel_err(got.cpu().numpy()[hit], want[hit])
    print(f"{name}: largest relative difference of the fused sums {err:.2e}")
    assert err <= REL


@pytest.mark.parametrize("name", ["cube16", "aniso", "tbct"])
def test_fast_sums_sart_and_solver(name, oracle_built):
    """The SART pass and the solver with fused sums stay within 1e-5 of the
    exact engine's volume (relative to its maximum)."""
    import gpu_b200
    cfg = SCANS[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    rng = np.random.default_rng(9)
    truth = rng.uniform(0, 0.05, o.vol_shape).astype(np.float32)
    b = torch.from_numpy(np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])).cuda()
    out = {}
    for fast in (False, True):
        g = gpu_b200.Geometry(ctr_desc(cfg, fast_sums=fast))
        v = torch.zeros(o.vol_shape, device="cuda")
        g.sart_pass(v, b, 0.8)
        s = gpu_b200.Solver(g, gpu_b200.F32, beta=0.3, lambda_tv=0.05, fgp_iters=4, objective=True)
        s.set_sinogram(b)
        s.set_volume(None)
        objs = s.iterate(3)
        x = torch.zeros(o.vol_shape, device="cuda")
        s.get_volume(x)
        out[fast] = (v.cpu().numpy(), x.cpu().numpy(), objs)
    for k in (0, 1):
        scale = np.abs(out[False][k]).max()
        assert np.abs(out[True][k] - out[False][k]).max() <= REL * scale
    np.testing.assert_allclose(out[True][2][:, 1], out[False][2][:, 1], rtol=1e-3)   # residuals cancel


def test_fast_sums_full_size():
    """512^3 / 1024x768: three views of the fused projector against the exact one."""
    import gpu_b200
    d = dict(nx=512, ny=512, nz=512, vx=0.5, nu=1024, nv=768, du=0.4, dso=1000.0, dod=-500.0, n_views=1024)
    args = (d["nx"], d["ny"], d["nz"], d["vx"], d["nu"], d["nv"], d["du"], d["dso"], d["dod"], d["n_views"])
    exact = gpu_b200.Geometry(gpu_b200.make_desc(*args))
    fast = gpu_b200.Geometry(gpu_b200.make_desc(*args, fast_sums=True))
    gen = torch.Generator(device="cuda").manual_seed(3)
    vol = torch.rand(exact.vol_shape, device="cuda", generator=gen) + 0.01
    for j in (0, 333, 700):
        a = torch.zeros((1,) + exact.view_shape, device="cuda")
        f = torch.zeros_like(a)
        exact.forward(vol, a, j, 1)
        fast.forward(vol, f, j, 1)
        hit = a > 0
        assert torch.equal(f > 0, hit)
        err = float(((f - a).abs()[hit] / a[hit]).max())
        assert err <= REL, f"view {j}: {err:.2e}"
