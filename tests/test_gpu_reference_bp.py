"""CTR_SART_REFERENCE_BP: the SART update with the reference backprojector's
own arithmetic (V63/kernel_IterativeRecon_universal.cu:571-810; for the
tetrahedron beam its program's backprojection and update).  With it a FP32
SART pass -- and the SART + FISTA + FGP-TV loop built on it -- equals the
reference's bit for bit: against the C restatement (pinned to the reference's
kernels compiled for the CPU) and against the golden fixtures made by those
kernels themselves."""
import os

import numpy as np
import pytest

from scan_configs import SMALL, STYLES, TBCT, ctr_desc, og_desc_xyz

CASES = dict(SMALL, **STYLES, **TBCT)
HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def flags(tiled=False):
    import gpu_b200
    return gpu_b200.SART_REFERENCE_BP | (gpu_b200.SART_TILED if tiled else 0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_sart_pass_equals_reference_golden(name):
    """From zero, on the golden sinogram: the reference's own SART pass output."""
    import gpu_b200
    cfg = CASES[name]
    gold = dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))
    g = gpu_b200.Geometry(ctr_desc(cfg))
    b = torch.from_numpy(gold["b"]).cuda()
    for tiled in (False, True):
        x = torch.zeros(g.vol_shape, device="cuda")
        g.sart_pass(x, b, 0.8, flags=flags(tiled))
        np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(gold["sart"]), err_msg=f"tiled={tiled}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_sart_pass_equals_restatement_from_signed_zeros(name, oracle_built):
    """From a volume of random values with -0 planted (the reference's "+= 0"
    turns them into +0 where no ray updates the voxel), two passes."""
    import gpu_b200
    cfg = CASES[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    g = gpu_b200.Geometry(ctr_desc(cfg))
    rng = np.random.default_rng(31)
    vol = rng.uniform(0, 0.05, o.vol_shape).astype(np.float32)
    vol[rng.uniform(size=vol.shape) < 0.2] = -0.0     # the tetrahedron beam's update has no "+= 0"
    b = np.stack([o.forward_view(vol * 1.1, j, 0) for j in range(cfg["nviews"])])
    want = o.sart_pass_ref(o.sart_pass_ref(vol, b, 0.8), b, 0.8)
    x = torch.from_numpy(vol).cuda()
    g.sart_pass(x, torch.from_numpy(b).cuda(), 0.8, flags=flags())
    g.sart_pass(x, torch.from_numpy(b).cuda(), 0.8, flags=flags())
    np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(want))


@pytest.mark.parametrize("name", ["cube16", "odd", "fan_slices_odd", "parallel", "tbct"])
def test_every_launch_shape_gives_the_same_result(name, oracle_built):
    import gpu_b200
    cfg = CASES[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    g = gpu_b200.Geometry(ctr_desc(cfg))
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02]]))
    b = torch.from_numpy(np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])).cuda()
    ref = None
    for bs in range(-1, g.BP_SHAPES):
        g.set_shapes(1, bs)
        x = torch.zeros(g.vol_shape, device="cuda")
        g.sart_pass(x, b, 0.8, flags=flags(bs % 2 == 0))
        got = bits(x.cpu().numpy())
        if ref is None:
            ref = got
        np.testing.assert_array_equal(got, ref, err_msg=f"bp shape {bs}")


@pytest.mark.parametrize("name", ["aniso", "tbct"])
def test_solver_equals_reference_call_sequence(name, oracle_built):
    """Three SART + FISTA + FGP-TV iterations (graph-captured) with the
    reference backprojector: the reference's loop restated, bit for bit."""
    import gpu_b200
    cfg = CASES[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    g = gpu_b200.Geometry(ctr_desc(cfg))
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]]))
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    beta, lam, it = np.float32(0.8), 0.05, 5
    s = gpu_b200.Solver(g, gpu_b200.F32, beta=float(beta), lambda_tv=lam, fgp_iters=it, fista=True, objective=True,
                        use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    s.set_sinogram(torch.from_numpy(b).cuda())
    s.set_volume(None)
    s.iterate(3)
    out = torch.zeros(o.vol_shape, device="cuda")
    s.get_volume(out)
    y = np.zeros(o.vol_shape, np.float32)
    xprev = np.zeros_like(y)
    t = np.float32(1.0)
    for _ in range(3):                       # V63/main_recon.cu:344-386
        x = o.fgp(o.sart_pass_ref(y, b, beta), beta * np.float32(lam), it)
        t_k = (np.float32(1.0) + np.sqrt(np.float32(1.0) + np.float32(4.0) * t * t, dtype=np.float32)) / np.float32(2.0)
        y, xprev = o.fista_momentum(y, xprev, x, t, t_k)
        t = np.float32(t_k)
    np.testing.assert_array_equal(bits(out.cpu().numpy()), bits(xprev))

