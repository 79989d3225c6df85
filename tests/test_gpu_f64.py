"""The FP64 reference solver (``vol_dtype=F64``) against the FP64 oracle's
call sequence (SART pass with the traversal's segments scattered, FGP-TV,
FISTA; everything in double on the CPU).  The GPU gathers the geometric chord
of every (voxel, ray) pair instead of scattering segments, so the two agree to
double rounding, not bit for bit."""
import numpy as np
import pytest

from scan_configs import CONFIG0, MIXED, ctr_desc, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def ellipsoid_problem(oracle_mod, cfg, n_ell, seed=100):
    o = oracle_mod.Oracle(og_desc_xyz(cfg))
    rng = np.random.default_rng(seed)
    params = oracle_mod.random_ellipsoids(rng, n_ell, 40.0, (5.0, 40.0), (0.01, 0.03))
    truth = o.phantom(params)
    b = o.phantom_sinogram(params)
    b = (b + 0.005 * b.max() * rng.standard_normal(b.shape)).astype(np.float32)
    return o, truth, b


def oracle_fista64(o, b, beta, lam_tv, fgp_iters, n):
    """V63/main_recon.cu:344-386 in FP64 with the solver's float parameters widened."""
    beta64 = float(np.float32(beta))
    lam64 = beta64 * float(np.float32(lam_tv))
    y = np.zeros(o.vol_shape)
    xprev = np.zeros(o.vol_shape)
    t = 1.0
    b64 = b.astype(np.float64)
    for _ in range(n):
        x = o.sart_pass_f64(y, b64, beta64)
        if lam_tv > 0:
            x = o.fgp_f64(x, lam64, fgp_iters)
        tk = (1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
        y = x + (t - 1.0) / tk * (x - xprev)
        xprev = x
        t = tk
    return xprev


def run_f64(cfg, b, beta, lam_tv, fgp_iters, n, objective=False):
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(cfg))
    s = gpu_b200.Solver(g, gpu_b200.F64, beta=beta, lambda_tv=lam_tv, fgp_iters=fgp_iters, fista=True,
                        objective=objective)
    s.set_sinogram(torch.from_numpy(b).cuda())
    s.set_volume(None)
    objs = s.iterate(n)
    out = torch.zeros(g.vol_shape, device="cuda", dtype=torch.float64)
    s.get_volume(out)
    return out.cpu().numpy(), objs, s


@pytest.mark.parametrize("cfg_name,n_ell,iters", [("mixed", 10, 3), ("config0", 10, 1)])
def test_f64_solver_matches_fp64_oracle(cfg_name, n_ell, iters, oracle_built):
    cfg = {"mixed": MIXED, "config0": CONFIG0}[cfg_name]
    o, truth, b = ellipsoid_problem(oracle_built, cfg, n_ell)
    beta, lam, fgp = 0.0625, 2e-4, 20
    want = oracle_fista64(o, b, beta, lam, fgp, iters)
    got, _, _ = run_f64(cfg, b, beta, lam, fgp, iters)
    err = np.abs(got - want).max() / truth.max()
    print(f"{cfg_name}: FP64 solver vs FP64 oracle after {iters} iterations: max error {err:.3e} of max attenuation")
    assert err <= 1e-10


def test_f64_objective(oracle_built):
    o, truth, b = ellipsoid_problem(oracle_built, MIXED, 10)
    got, objs, s = run_f64(MIXED, b, 0.0625, 2e-4, 20, 2, objective=True)
    ax = np.stack([o.forward_view_f64(got, j) for j in range(b.shape[0])])
    fid = float(np.sum((ax - b.astype(np.float64)) ** 2))
    np.testing.assert_allclose(objs[-1, 1], fid, rtol=1e-9)
    assert s.iteration == 2
    x32 = torch.zeros(got.shape, device="cuda")
    s.get_volume_f32(x32)
    np.testing.assert_array_equal(x32.cpu().numpy(), got.astype(np.float32))


def test_f64_refusals():
    import gpu_b200
    from scan_configs import STYLES
    g = gpu_b200.Geometry(ctr_desc(STYLES["parallel"]))
    with pytest.raises(gpu_b200.CtrError):
        gpu_b200.Solver(g, gpu_b200.F64, beta=0.1)
    g0 = gpu_b200.Geometry(ctr_desc(MIXED))
    s = gpu_b200.Solver(g0, gpu_b200.F64, beta=0.1)
    with pytest.raises(gpu_b200.CtrError):
        s.set_slabs(2)
    with pytest.raises(gpu_b200.CtrError):
        gpu_b200.Batch([g0], gpu_b200.F64)
