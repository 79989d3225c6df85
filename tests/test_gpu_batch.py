"""Batched reconstruction of scans of uneven sizes (``ctr_batch``): one CUDA
graph launch per iteration runs every scan's SART pass, FGP-TV, FISTA step and
objective.  Each scan's result must be bit-identical to the single-scan solver
on the same inputs, which is itself pinned to the oracle's call sequence."""
import numpy as np
import pytest

from scan_configs import SMALL, TBCT, ctr_desc, og_desc_xyz

SCANS = dict(SMALL, **TBCT)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


PHANTOM = np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]])


def scans(oracle_mod):
    out = []
    for name in ["cube16", "odd", "fine", "aniso", "fine_even", "tbct"]:   # a tetrahedron-beam scan among them
        cfg = SCANS[name]
        o = oracle_mod.Oracle(og_desc_xyz(cfg))
        b = np.stack([o.forward_view(o.phantom(PHANTOM), j, 0) for j in range(cfg["nviews"])])
        out.append((cfg, torch.from_numpy(b).cuda()))
    return out


def bits(t):
    return t.float().cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("dtype", ["f32", "f16", "bf16_sr", "f16_refine"])
def test_batch_equals_single_solver(dtype, persistent, oracle_built):
    """bf16_sr: stochastic rounding, whose per-pass seed the batch reads from
    device memory; the single-scan solver issues those passes directly.
    persistent: the SART views of all scans in one persistent launch per
    iteration (ctr_batch_set_persistent), its blocks handed out as a data
    flow over the scans' phases, the same per-ray and per-voxel code."""
    import gpu_b200
    vdt = {"f32": gpu_b200.F32, "f16": gpu_b200.F16, "bf16_sr": gpu_b200.BF16, "f16_refine": gpu_b200.F16}[dtype]
    tdt = {"f32": torch.float32, "f16": torch.float16, "bf16_sr": torch.bfloat16, "f16_refine": torch.float16}[dtype]
    data = scans(oracle_built)
    flags = gpu_b200.SART_STOCHASTIC_ROUND if dtype.endswith("_sr") else 0
    kw = dict(beta=0.8, lambda_tv=0.05, fgp_iters=4, fista=True, objective=True, sart_flags=flags,
              refine=dtype.endswith("_refine"))
    geoms = [gpu_b200.Geometry(ctr_desc(cfg)) for cfg, _ in data]
    batch = gpu_b200.Batch(geoms, vdt, **kw)
    if persistent:
        batch.set_persistent(True)
    for i, (_, b) in enumerate(data):
        batch.set_sinogram(i, b)
    batch.reset()
    objs = np.concatenate([batch.iterate(2), batch.iterate(1)], axis=1)
    for i, (cfg, b) in enumerate(data):
        g1 = gpu_b200.Geometry(ctr_desc(cfg))
        s = gpu_b200.Solver(g1, vdt, use_graph=True, **kw)
        s.set_sinogram(b)
        s.set_volume(None)
        ref_obj = s.iterate(3)
        want = torch.zeros((cfg["nz"], cfg["ny"], cfg["nx"]), device="cuda", dtype=tdt)
        got = torch.zeros_like(want)
        s.get_volume(want)
        batch.get_volume(i, got)
        np.testing.assert_array_equal(bits(got), bits(want))
        np.testing.assert_array_equal(objs[i], ref_obj)
        assert objs[i, -1, 1] < objs[i, 0, 1]


def test_persistent_batch_refusals(oracle_built):
    """The persistent pass runs the engine's update with the reference's sums:
    the reference backprojection arithmetic is refused, and the per-view form
    comes back with set_persistent(False)."""
    import gpu_b200
    data = scans(oracle_built)[:2]
    geoms = [gpu_b200.Geometry(ctr_desc(cfg)) for cfg, _ in data]
    batch = gpu_b200.Batch(geoms, gpu_b200.F32, beta=0.8, sart_flags=gpu_b200.SART_REFERENCE_BP)
    with pytest.raises(gpu_b200.CtrError):
        batch.set_persistent(True)
    batch.set_persistent(False)


def test_batch_reset_and_workspace_growth(oracle_built):
    """A geometry's workspace reallocated by another call between iterations
    (the adjoint needs larger ray records) makes the batch capture again."""
    import gpu_b200
    data = scans(oracle_built)[:3]
    geoms = [gpu_b200.Geometry(ctr_desc(cfg)) for cfg, _ in data]
    batch = gpu_b200.Batch(geoms, gpu_b200.F32, beta=0.8, lambda_tv=0.05, fgp_iters=3)
    for i, (_, b) in enumerate(data):
        batch.set_sinogram(i, b)
    batch.reset()
    first = batch.iterate(2)
    batch.reset()
    batch.iterate(1)
    cfg, b = data[1]
    vol = torch.zeros((cfg["nz"], cfg["ny"], cfg["nx"]), device="cuda")
    geoms[1].backproject(b, vol)                       # grows geometry 1's ray workspace
    second = batch.iterate(1)
    np.testing.assert_array_equal(second[:, 0], first[:, 1])


def test_batch_rejects_shared_geometry():
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(SMALL["cube16"]))
    with pytest.raises(gpu_b200.CtrError):
        gpu_b200.Batch([g, g], gpu_b200.F32)
