"""Mixed precision (BF16/FP16 storage, FP32 arithmetic) against the FP64
oracle: SART + FISTA + FGP-TV iterations on a seeded 10-ellipsoid phantom
whose sinogram is the FP64 analytic line integrals plus 0.5 % noise.  RMSE is
stated relative to the phantom's maximum attenuation.

Two relaxations: 0.8 (5 iterations) and the reference's FISTA step
2/Lip_con = 0.0625 (V63/main_recon.cu:58,161; 5 and 20 iterations).  With
the small step each view's update is small against the stored value, so
rounding to FP16/BF16 storage loses more of it and the error grows with the
iteration count; the limits record that.  (0.8 under FISTA diverges after a
few iterations, the FP64 oracle included, so it is not run longer.)"""
import numpy as np
import pytest

from scan_configs import MIXED, ctr_desc, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

LAM_TV, FGP = 2e-4, 20

# (relaxation, iterations, storage mode, RMSE limit relative to max attenuation)
CASES = [(0.8, 5, "f32", 1e-4), (0.8, 5, "f16", 1e-3), (0.8, 5, "f16_sr", 1e-3), (0.8, 5, "bf16_sr", 4e-3),
         (0.8, 5, "bf16", 8e-3),
         (0.0625, 5, "f32", 1e-4), (0.0625, 5, "f16", 1e-3), (0.0625, 5, "f16_sr", 1e-3),
         (0.0625, 5, "bf16_sr", 8e-3), (0.0625, 5, "bf16", 1.6e-2),
         (0.0625, 20, "f32", 2e-4), (0.0625, 20, "f16", 6e-3), (0.0625, 20, "f16_sr", 4e-3),
         (0.0625, 20, "bf16_sr", 2.5e-2), (0.0625, 20, "bf16", 6e-2)]


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
    return o, truth, b, {}


def fp64_reference(problem, beta, iters):
    """FP64 oracle of the same call sequence (V63/main_recon.cu:344-386) after
    `iters` iterations; each relaxation's run continues from its last state."""
    o, _, b, cache = problem
    if beta not in cache:
        cache[beta] = dict(n=0, y=np.zeros(o.vol_shape), xprev=np.zeros(o.vol_shape), t=1.0)
    st = cache[beta]
    assert st["n"] <= iters, "iteration counts of one relaxation are requested in increasing order"
    while st["n"] < iters:
        x = o.sart_pass_f64(st["y"], b.astype(np.float64), beta)
        x = o.fgp_f64(x, beta * LAM_TV, FGP)
        tk = (1.0 + np.sqrt(1.0 + 4.0 * st["t"] * st["t"])) / 2.0
        st["y"] = x + (st["t"] - 1.0) / tk * (x - st["xprev"])
        st["xprev"] = x
        st["t"] = tk
        st["n"] += 1
    return st["xprev"]


def run(b, vdt, beta, iters, flags=0):
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(MIXED))
    tdt = {gpu_b200.F32: torch.float32, gpu_b200.F16: torch.float16, gpu_b200.BF16: torch.bfloat16}[vdt]
    s = gpu_b200.Solver(g, vdt, beta=beta, lambda_tv=LAM_TV, fgp_iters=FGP, fista=True, objective=False,
                        sart_flags=flags)
    sino = torch.from_numpy(b).cuda().to(tdt)
    s.set_sinogram(sino)
    s.set_volume(None)
    s.iterate(iters)
    out = torch.zeros(g.vol_shape, device="cuda", dtype=tdt)
    s.get_volume(out)
    return out.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("beta,iters,mode,limit", CASES)
def test_rmse_against_fp64_oracle(problem, beta, iters, mode, limit):
    import gpu_b200
    _, truth, b, _ = problem
    ref = fp64_reference(problem, beta, iters)
    vdt = {"f32": gpu_b200.F32, "f16": gpu_b200.F16, "f16_sr": gpu_b200.F16, "bf16": gpu_b200.BF16,
           "bf16_sr": gpu_b200.BF16}[mode]
    flags = gpu_b200.SART_STOCHASTIC_ROUND if mode.endswith("_sr") else 0
    got = run(b, vdt, beta, iters, flags)
    mu_max = float(truth.max())
    rmse = float(np.sqrt(np.mean((got - ref) ** 2))) / mu_max
    maxerr = float(np.abs(got - ref).max()) / mu_max
    print(f"beta {beta}, {iters} iterations, {mode}: RMSE {rmse:.3e}, max abs error {maxerr:.3e} "
          f"(relative to max attenuation {mu_max:.4f})")
    assert rmse <= limit
