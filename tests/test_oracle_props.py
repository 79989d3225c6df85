"""Properties of the CPU oracle itself (no GPU): the FP64 twin agrees with the
FP32 restatement, the scatter adjoint is the projector's transpose, analytic
line integrals agree with the Siddon projection of the voxelised phantom, the
spatial ramp kernel equals the padded-DFT filter, FGP decreases its
objective, and the reference's FISTA loop is stable at its own step."""
import numpy as np
import pytest

from scan_configs import FISTA32, MIXED, SMALL, og_desc_xyz


@pytest.fixture(scope="module")
def omix(oracle_built):
    return oracle_built.Oracle(og_desc_xyz(MIXED))


def test_fp64_twin_agrees_with_fp32(omix):
    """FP32 Siddon sums against the FP64 traversal: ~3e-5 of the maximum ray
    sum on a white-noise volume (alpha rounding at ~200 segment boundaries)."""
    rng = np.random.default_rng(1)
    vol = rng.uniform(0, 1, omix.vol_shape).astype(np.float32)
    for j in (0, 17, 45):
        a = omix.forward_view(vol, j, 0).astype(np.float64)
        b = omix.forward_view_f64(vol.astype(np.float64), j)
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


def test_scatter_adjoint_is_transpose(omix):
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 1, omix.vol_shape).astype(np.float32)
    for j in (3, 30):
        y = rng.standard_normal(omix.view_shape).astype(np.float32)
        ax = omix.forward_view(x, j, 0).astype(np.float64)
        aty = omix.adjoint_view(y, j)
        lhs, rhs = float(np.sum(ax * y)), float(np.sum(aty * x))
        assert abs(lhs - rhs) <= 1e-5 * np.sqrt(np.sum(ax * ax) * np.sum(y.astype(np.float64) ** 2))


def test_analytic_projection_matches_voxelised(omix, oracle_built):
    params = np.array([[3.0, -2.0, 1.0, 40.0, 30.0, 25.0, 0.3, 0.5, 0.1, 0.02]])
    vol = omix.phantom(params)
    for j in (0, 20):
        fp = omix.forward_view(vol, j, 0)
        an = omix.phantom_sinogram(params, [j])[0]
        inside = an > 0.5 * an.max()
        assert np.abs(fp[inside] - an[inside]).mean() <= 0.02 * an.max()


def test_ramp_kernel_is_the_padded_dft_filter(oracle_built):
    o = oracle_built.Oracle(og_desc_xyz(SMALL["cube16"]))
    rng = np.random.default_rng(3)
    rows = rng.standard_normal((5, 24)).astype(np.float32)
    a = o.ramp_filter(rows)
    b = o.ramp_filter(rows, dft=True)
    assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


def test_fgp_decreases_its_objective(oracle_built):
    cfg = SMALL["cube16"]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    rng = np.random.default_rng(4)
    f = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    lam = 0.05

    def obj(x):
        return 0.5 * np.sum((x.astype(np.float64) - f) ** 2) + lam * o.tv_norm(x)

    x = o.fgp(f, lam, 20)
    assert obj(x) < obj(f)
    x2 = o.fgp(f, lam, 40)
    assert obj(x2) <= obj(x) * (1 + 1e-4)


def test_fista_step_of_the_reference_is_stable(oracle_built):
    """The reference's loop (V63/main_recon.cu:344-386) in FP64: SART from y,
    FGP-TV with lambda = beta * lambda_TV, FISTA momentum.  At its own step
    beta = 2/Lip_con = 2/32 (:58,161) the error against the phantom stays
    bounded for 30 iterations; at beta = 0.8, the plain-SART relaxation, the
    momentum amplifies it geometrically (RMSE ~300x the phantom's maximum by
    iteration 30 on this scan)."""
    o = oracle_built.Oracle(og_desc_xyz(FISTA32))
    rng = np.random.default_rng(100)
    params = oracle_built.random_ellipsoids(rng, 10, 40.0, (5.0, 40.0), (0.01, 0.03))
    truth = o.phantom(params)
    b = o.phantom_sinogram(params)
    b = (b + 0.005 * b.max() * rng.standard_normal(b.shape)).astype(np.float64)
    mu = float(truth.max())

    def rmse_history(beta, iters=30):
        y = np.zeros(o.vol_shape)
        xprev = np.zeros_like(y)
        t = 1.0
        out = []
        for _ in range(iters):
            x = o.fgp_f64(o.sart_pass_f64(y, b, beta), beta * 2e-4, 20)
            tk = (1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
            y = x + (t - 1.0) / tk * (x - xprev)
            xprev = x
            t = tk
            out.append(float(np.sqrt(np.mean((x - truth) ** 2))) / mu)
        return out

    small = rmse_history(2.0 / 32.0)
    assert max(small) < 0.1 and small[-1] < 0.06
    large = rmse_history(0.8)
    assert large[-1] > 10.0 and large[-1] > 4.0 * large[-5]
