"""Mixed precision (BF16/FP16 storage, FP32 arithmetic) against the FP64
oracle: 5 SART + FISTA + FGP-TV iterations on a seeded 10-ellipsoid phantom
whose sinogram is the FP64 analytic line integrals plus 0.5 % noise.  RMSE is
stated relative to the phantom's maximum attenuation."""
import numpy as np
import pytest

from scan_configs import MIXED, ctr_desc, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ITERS, BETA, LAM_TV, FGP = 5, 0.8, 2e-4, 20


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def problem(oracle_built):
    o = oracle_built.Oracle(og_desc_xyz(MIXED))
    rng = np.random.default_rng(100)
    params = oracle_built.random_ellipsoids(rng, 10, 40.0, (5.0, 40.0), (0.01, 0.03))
    truth = o.phantom(params)
    b = o.phantom_sinogram(params)
    b = (b + 0.005 * b.max() * rng.standard_normal(b.shape)).astype(np.float32)
    # FP64 oracle of the same call sequence (V63/main_recon.cu:344-386)
    y = np.zeros(o.vol_shape)
    xprev = np.zeros_like(y)
    t = 1.0
    for _ in range(ITERS):
        x = o.sart_pass_f64(y, b.astype(np.float64), BETA)
        x = o.fgp_f64(x, BETA * LAM_TV, FGP)
        tk = (1.0 + np.sqrt(1.0 + 4.0 * t * t)) / 2.0
        y = x + (t - 1.0) / tk * (x - xprev)
        xprev = x
        t = tk
    return o, truth, b, xprev


def run(b, vdt, flags=0):
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(MIXED))
    tdt = {gpu_b200.F32: torch.float32, gpu_b200.F16: torch.float16, gpu_b200.BF16: torch.bfloat16}[vdt]
    s = gpu_b200.Solver(g, vdt, beta=BETA, lambda_tv=LAM_TV, fgp_iters=FGP, fista=True, objective=False,
                        sart_flags=flags)
    sino = torch.from_numpy(b).cuda().to(tdt)
    s.set_sinogram(sino)
    s.set_volume(None)
    s.iterate(ITERS)
    out = torch.zeros(g.vol_shape, device="cuda", dtype=tdt)
    s.get_volume(out)
    return out.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("mode,limit", [("f32", 1e-4), ("f16", 1e-3), ("f16_sr", 1e-3), ("bf16_sr", 4e-3),
                                        ("bf16", 8e-3)])
def test_rmse_against_fp64_oracle(problem, mode, limit):
    import gpu_b200
    o, truth, b, ref = problem
    vdt = {"f32": gpu_b200.F32, "f16": gpu_b200.F16, "f16_sr": gpu_b200.F16, "bf16": gpu_b200.BF16,
           "bf16_sr": gpu_b200.BF16}[mode]
    flags = gpu_b200.SART_STOCHASTIC_ROUND if mode.endswith("_sr") else 0
    got = run(b, vdt, flags)
    mu_max = float(truth.max())
    rmse = float(np.sqrt(np.mean((got - ref) ** 2))) / mu_max
    maxerr = float(np.abs(got - ref).max()) / mu_max
    print(f"{mode}: RMSE {rmse:.3e}, max abs error {maxerr:.3e} (relative to max attenuation {mu_max:.4f})")
    assert rmse <= limit
