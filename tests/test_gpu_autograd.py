"""torch.autograd over the C ABI (gpu_b200.autograd) on the differentiation
scan: 256^3, 360 views, 384^2 detector.  Loss 0.5||Ax - b||^2 + 1e-3 TV_iso(x)."""
import numpy as np
import pytest

from scan_configs import CONFIG2, SMALL, ctr_desc, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def scan2():
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(CONFIG2))
    rng = np.random.default_rng(2)
    params = np.zeros((12, 10))
    params[:, 0:3] = rng.uniform(-30, 30, (12, 3))
    params[:, 3:6] = rng.uniform(5, 30, (12, 3))
    params[:, 6:9] = rng.uniform(0, 2 * np.pi, (12, 3))
    params[:, 9] = rng.uniform(0.01, 0.03, 12)
    truth = torch.zeros(g.vol_shape, device="cuda")
    g.phantom_voxelize(params, truth)
    b = torch.zeros((CONFIG2["nviews"],) + g.view_shape, device="cuda")
    g.forward(truth, b)
    return g, truth, b


def test_function_pair_is_the_engine(scan2):
    from gpu_b200.autograd import BackProject, ForwardProject
    g, truth, b = scan2
    x = truth.clone().requires_grad_(True)
    y = ForwardProject.apply(x, g, 0, 16)
    ref = torch.zeros_like(y)
    g.forward(truth, ref, 0, 16)
    assert torch.equal(y.detach(), ref)
    w = torch.randn_like(y)
    (y * w).sum().backward()
    ref_g = torch.zeros_like(truth)
    g.backproject(w.contiguous(), ref_g, 0, 16)
    assert torch.equal(x.grad, ref_g)
    s = w.clone().requires_grad_(True)
    z = BackProject.apply(s, g, 0, 16)
    assert torch.equal(z.detach(), ref_g)


def test_dot_product_16_pairs(scan2):
    """16 seeded (x, y): x ~ U[0,1] over voxels, y ~ N(0,1) over detector bins."""
    g, _, _ = scan2
    gen = torch.Generator(device="cuda").manual_seed(16)
    for _ in range(16):
        x = torch.rand(g.vol_shape, device="cuda", generator=gen)
        y = torch.randn((CONFIG2["nviews"],) + g.view_shape, device="cuda", generator=gen)
        a, c = g.dot_test(x, y)
        assert abs(a - c) <= 1e-6 * max(abs(a), abs(c)), (a, c)


def test_gradient_finite_differences(scan2):
    """Central differences, h = 1e-3, at 64 seeded voxels inside the object.
    The loss is quadratic + TV, so the difference quotient has no truncation
    error in the data term; what remains is FP32 rounding of the projections,
    hence the stated 2e-2 relative tolerance."""
    from gpu_b200.autograd import recon_loss
    g, truth, b = scan2
    gen = torch.Generator(device="cuda").manual_seed(7)
    x0 = (truth * 0.7 + 0.002 * torch.rand(truth.shape, device="cuda", generator=gen)).contiguous()
    x = x0.clone().requires_grad_(True)
    loss = recon_loss(x, b, g, 1e-3, chunk=64)
    loss.backward()
    grad = x.grad
    rng = np.random.default_rng(64)
    idx = np.argwhere(truth.cpu().numpy() > 0)
    pick = idx[rng.choice(len(idx), 64, replace=False)]
    h = 1e-3
    bad = []
    with torch.no_grad():
        for (k, j, i) in pick:
            xp = x0.clone(); xp[k, j, i] += h
            xm = x0.clone(); xm[k, j, i] -= h
            fd = (recon_loss(xp, b, g, 1e-3, 64) - recon_loss(xm, b, g, 1e-3, 64)).item() / (2 * h)
            an = grad[k, j, i].item()
            if abs(fd - an) > 2e-2 * max(abs(an), 1e-3 * grad.abs().max().item()):
                bad.append((int(k), int(j), int(i), an, fd))
    assert not bad, bad[:5]


def test_gradient_vs_fp64_oracle(oracle_built):
    """The data-term gradient A^T(Ax - b) against the FP64 oracle's, on a scan
    without degenerate rays."""
    import gpu_b200
    from gpu_b200.autograd import data_fidelity_loss
    cfg = SMALL["fine_even"]
    g = gpu_b200.Geometry(ctr_desc(cfg))
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, o.vol_shape)
    b = rng.uniform(0, 5, (cfg["nviews"],) + o.view_shape)
    xt = torch.tensor(x, dtype=torch.float32, device="cuda", requires_grad=True)
    loss = data_fidelity_loss(xt, torch.tensor(b, dtype=torch.float32, device="cuda"), g, chunk=5)
    loss.backward()
    got = xt.grad.cpu().numpy().astype(np.float64)
    x32 = x.astype(np.float32).astype(np.float64)
    ref = np.zeros_like(x)
    for j in range(cfg["nviews"]):
        r = o.forward_view_f64(x32, j) - b[j].astype(np.float32)
        ref += o.adjoint_view_f64(r, j)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


def test_fifty_step_reconstruction(scan2):
    """50 gradient steps on 0.5||Ax-b||^2 + 1e-3 TV with 64-view chunk
    recomputation; step 1/L from power iteration on A^T A."""
    from gpu_b200.autograd import recon_loss
    g, truth, b = scan2
    v = torch.ones(g.vol_shape, device="cuda")
    sino = torch.zeros_like(b)
    for _ in range(8):
        g.forward(v, sino)
        g.backproject(sino, v)
        lip = v.norm().item()
        v /= lip if lip > 0 else 1.0
    step = 1.0 / lip
    x = torch.zeros_like(truth, requires_grad=True)
    losses = []
    for _ in range(50):
        loss = recon_loss(x, b, g, 1e-3, chunk=64)
        losses.append(loss.item())
        (gx,) = torch.autograd.grad(loss, x)
        with torch.no_grad():
            x -= step * gx
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.05 * losses[0]
    err0 = truth.norm().item()
    assert (x.detach() - truth).norm().item() < 0.6 * err0


def test_fidelity_gradient_of_the_measured_data():
    """d/db 0.5||Ax - b||^2 = -(Ax - b), alongside the volume's gradient."""
    import gpu_b200
    from gpu_b200.autograd import data_fidelity_loss
    cfg = SMALL["cube16"]
    g = gpu_b200.Geometry(ctr_desc(cfg))
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(g.vol_shape, device="cuda", generator=gen).requires_grad_(True)
    b = torch.rand((cfg["nviews"],) + g.view_shape, device="cuda", generator=gen).requires_grad_(True)
    loss = data_fidelity_loss(x, b, g, chunk=5)
    (2.0 * loss).backward()
    ax = torch.zeros_like(b)
    g.forward(x.detach(), ax)
    torch.testing.assert_close(b.grad, -2.0 * (ax - b.detach()), rtol=0, atol=0)
    ref = torch.zeros_like(x)
    g.backproject((ax - b.detach()).contiguous(), ref)
    torch.testing.assert_close(x.grad, 2.0 * ref, rtol=1e-6, atol=1e-6 * float(ref.abs().max()))
