"""The z-slab SART of the reference's multi-GPU build on the GPU.

Per slab and view, the library's partial projection, ordered combination and
slab update (ctr_forward_partial, ctr_combine_partials, ctr_sart_update)
against the reference's multi-GPU kernels (golden fixtures,
tests/golden/make_golden_slabs.py) and the oracle; the whole D-slab pass on
one GPU (ctr_sart_pass_slabs) and the reference-compatible
Reconstruction_3D_ray_driven_CBCT with ctr_set_default_devices(D), linear and
tiled; the 512^3 scan split in 4; the one-slab-per-rank driver
(gpu_b200/slabs.py) over a one-rank NCCL group.  Bit-exact throughout.
"""
import os

import numpy as np
import pytest

from scan_configs import SLABS, ctr_desc, og_desc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(name, D) for name, cfg in SLABS.items() for D in cfg["slabs"]]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"slabs_{name}.npz")))


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def slab_geoms(cfg, D):
    import gpu_b200
    return [gpu_b200.Geometry(ctr_desc(cfg), D, s) for s in range(D)]


@pytest.mark.parametrize("name,D", CASES)
def test_per_view_steps_equal_reference(name, D, oracle_built):
    """Partial sums and correction of one view, then each slab's update with
    the multi-GPU backprojector's arithmetic (golden) and with the engine's
    gather update (oracle), linear and tiled."""
    import gpu_b200
    cfg = SLABS[name]
    g = load(name)
    j = int(g["view"])
    zs = cfg["nz"] // D
    gs = slab_geoms(cfg, D)
    assert [x.slab_info() for x in gs] == [(D, s, zs * s) for s in range(D)]
    rows, nu = gs[0].view_shape
    for tiled in (False, True):
        parts = torch.zeros((D, rows, nu, 2), device="cuda")
        vols = []
        for s, gg in enumerate(gs):
            v = dev(g["vol0"][zs * s:zs * (s + 1)])
            if tiled:
                t = torch.zeros(gg.tiled_count(), device="cuda")
                gg.volume_tiling(v, t, True)
                v = t
            vols.append(v)
            gg.forward_partial(v, j, parts[s], gpu_b200.VOLUME_TILED if tiled else 0)
        p = parts.cpu().numpy()
        np.testing.assert_array_equal(bits(p[..., 0]), bits(g[f"w_{D}"]), err_msg=f"tiled={tiled}")
        np.testing.assert_array_equal(bits(p[..., 1]), bits(g[f"l_{D}"]), err_msg=f"tiled={tiled}")
        rays = torch.zeros((rows, nu, 2), device="cuda")
        gs[0].combine_partials(parts, j, dev(g["b"][j]), rays)
        np.testing.assert_array_equal(bits(rays[..., 0].cpu().numpy()), bits(g[f"corr_{D}"]))
        for ref_bp in (True, False):
            out = []
            for s, gg in enumerate(gs):
                v = vols[s].clone()
                fl = (gpu_b200.SART_REFERENCE_BP if ref_bp else 0) | (gpu_b200.VOLUME_TILED if tiled else 0)
                gg.sart_update(v, rays, j, 0.8, fl)
                if tiled:
                    lin = torch.zeros(gg.vol_shape, device="cuda")
                    gg.volume_tiling(v, lin, False)
                    v = lin
                out.append(v.cpu().numpy())
            got = np.concatenate(out)
            if ref_bp:
                want = g[f"bp1_{D}"]
            else:
                d = og_desc(cfg)
                want = np.concatenate([
                    oracle_built.Oracle(oracle_built.slab_desc(d, D, s)).backproject_gather(
                        g["vol0"][zs * s:zs * (s + 1)], g[f"corr_{D}"], j, 0.8) for s in range(D)])
            np.testing.assert_array_equal(bits(got), bits(want), err_msg=f"tiled={tiled} reference_bp={ref_bp}")


@pytest.mark.parametrize("name,D", CASES)
def test_one_gpu_slab_pass(name, D, oracle_built):
    """ctr_sart_pass_slabs: the reference's D-device pass (golden), linear and
    tiled; with the engine's update, the oracle's D-slab pass."""
    import gpu_b200
    cfg = SLABS[name]
    g = load(name)
    geom = gpu_b200.Geometry(ctr_desc(cfg))
    b = dev(g["b"])
    for tiled in (False, True):
        x = dev(g["vol0"])
        geom.sart_pass_slabs(x, b, 0.8, D, flags=gpu_b200.SART_REFERENCE_BP | (gpu_b200.SART_TILED if tiled else 0))
        np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(g[f"sart_{D}"]), err_msg=f"tiled={tiled}")
    o = oracle_built.Oracle(og_desc(cfg))
    want = o.sart_pass_slabs(g["vol0"], g["b"], 0.8, D, engine=True)
    x = dev(g["vol0"])
    geom.sart_pass_slabs(x, b, 0.8, D, flags=gpu_b200.SART_TILED)
    np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(want))


@pytest.mark.parametrize("name,D", [("cone_wide", 4), ("fan_edges", 3), ("parallel_slabs", 2), ("tbct_slabs", 4)])
def test_reference_compatible_entry_point_with_devices(name, D, oracle_built, capfd):
    """Number_of_Devices = D: Reconstruction_3D_ray_driven_CBCT and
    Forward_3D_ray_driven_siddon return the D-device build's numbers; back at
    1 device, the one-device build's."""
    import gpu_b200
    cfg = SLABS[name]
    g = load(name)
    gpu_b200.set_default_geometry(ctr_desc(cfg))
    try:
        gpu_b200.set_default_devices(D)
        x = g["vol0"].copy()
        gpu_b200.reconstruction_3d_ray_driven_cbct(x, g["b"].copy(), 0.8)
        assert gpu_b200.last_error() == ""
        np.testing.assert_array_equal(bits(x), bits(g[f"sart_{D}"]))
        proj = np.zeros_like(g["b"])
        gpu_b200.forward_3d_ray_driven_siddon(g["vol0"].copy(), proj)
        assert gpu_b200.last_error() == ""
        np.testing.assert_array_equal(bits(proj[int(g["view"])]), bits(g[f"fwd_split_{D}"]))
        if cfg.get("ct_style", 0) != 3:   # T42's backprojector has no command 0 for the check
            gpu_b200.check_matched_joint_operator(g["vol0"].copy())   # the D-device check runs and prints
            assert gpu_b200.last_error() == ""
            assert "inner product" in capfd.readouterr().out
    finally:
        gpu_b200.set_default_devices(1)
    x = g["vol0"].copy()
    gpu_b200.reconstruction_3d_ray_driven_cbct(x, g["b"].copy(), 0.8)
    o = oracle_built.Oracle(og_desc(cfg))
    np.testing.assert_array_equal(bits(x), bits(o.sart_pass_ref(g["vol0"], g["b"], 0.8)))


def test_slab_geometry_errors():
    import gpu_b200
    cfg = SLABS["pitch07"]
    for D in (2, 4):                                           # 15 detector rows do not split
        with pytest.raises(gpu_b200.CtrError):
            gpu_b200.Geometry(ctr_desc(cfg), D, 0)
    with pytest.raises(gpu_b200.CtrError):                     # slab out of range
        gpu_b200.Geometry(ctr_desc(cfg), 3, 3)
    tb = dict(nx=16, ny=16, nz=16, nu=32, nv=4, nviews=4, vx=1.0, du=1.2, dso=40.0, dod=-40.0, ct_style=3,
              n_sources=2)
    with pytest.raises(gpu_b200.CtrError):                     # the tetrahedron beam: 16 slices in 3
        gpu_b200.Geometry(ctr_desc(tb), 3, 0)
    assert gpu_b200.Geometry(ctr_desc(tb), 2, 1).slab_info() == (2, 1, 8)   # its multi-GPU build's slab
    sg = gpu_b200.Geometry(ctr_desc(cfg), 3, 1)
    with pytest.raises(gpu_b200.CtrError):                     # the solver needs the whole volume
        gpu_b200.Solver(sg, gpu_b200.F32)
    full = gpu_b200.Geometry(ctr_desc(cfg))
    x = torch.zeros(full.vol_shape, device="cuda")
    b = torch.zeros((cfg["nviews"],) + full.view_shape, device="cuda")
    with pytest.raises(gpu_b200.CtrError):                     # 12 slices do not split in 5
        full.sart_pass_slabs(x, b, 0.8, 5)


SCAN = dict(nx=512, ny=512, nz=512, vx=0.5, nu=1024, nv=768, du=0.4, dso=1000.0, dod=-500.0, nviews=1024)


def test_full_size_four_slabs(oracle_built):
    """The 512^3 / 1024x768 / 1024-view scan split in 4 (the reference's
    default Number_of_Devices): one view of the slab pass from a non-zero
    volume, the multi-GPU backprojector's arithmetic and the engine's update,
    against the oracle."""
    import gpu_b200
    D = 4
    geom = gpu_b200.Geometry(gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"],
                                                SCAN["du"], SCAN["dso"], SCAN["dod"], SCAN["nviews"]))
    d = oracle_built.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["nu"], SCAN["nv"], SCAN["nviews"], SCAN["vx"],
                               SCAN["du"], SCAN["dso"], SCAN["dod"])
    o = oracle_built.Oracle(d)
    half = 0.5 * SCAN["nx"] * SCAN["vx"]
    p = oracle_built.random_ellipsoids(np.random.default_rng(512), 12, 0.5 * half, (0.05 * half, 0.6 * half),
                                       (0.01 / SCAN["vx"], 0.03 / SCAN["vx"]))
    vol = torch.zeros(geom.vol_shape, device="cuda")
    geom.phantom_voxelize(p, vol)
    h = vol.cpu().numpy()
    j = 333
    b = torch.zeros((SCAN["nviews"],) + geom.view_shape, device="cuda")
    geom.forward(vol * 1.05, b[j:j + 1], j, 1)
    bh = b.cpu().numpy()
    for flags, engine in ((gpu_b200.SART_REFERENCE_BP | gpu_b200.SART_TILED, False), (gpu_b200.SART_TILED, True)):
        x = vol.clone()
        geom.sart_pass_slabs(x, b, 0.8, D, j, 1, flags=flags)
        got = x.cpu().numpy()
        assert np.count_nonzero(got != h) > 0.05 * h.size
        want = o.sart_pass_slabs(h, bh, 0.8, D, v0=j, nv=1, engine=engine)
        np.testing.assert_array_equal(bits(got), bits(want), err_msg=f"engine={engine}")


def test_slab_driver_over_nccl_one_rank(oracle_built):
    """gpu_b200.slabs.SlabSART on the GPU with a one-rank NCCL group (the only
    group one GPU allows without ranks waiting on one another): the exchange
    is all_gather_into_tensor of one part, the combination of one part is the
    one-device correction, so the driver's pass equals ctr_sart_pass bit for
    bit (both update arithmetics, linear and tiled slab volume)."""
    import socket
    from datetime import timedelta

    import torch.distributed as dist

    import gpu_b200
    from gpu_b200.slabs import SlabOps, SlabSART
    cfg = SLABS["cone_wide"]
    g = load("cone_wide")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        ops = SlabOps(ctr_desc(cfg), 1, 0)
        drv = SlabSART(ops, 0, 1, "cuda")
        whole = gpu_b200.Geometry(ctr_desc(cfg))
        b = dev(g["b"])
        for flags in (gpu_b200.SART_REFERENCE_BP, 0):
            want = dev(g["vol0"])
            whole.sart_pass(want, b, 0.8, flags=flags)
            x = dev(g["vol0"])
            drv.views(x, b, 0.8, 0, cfg["nviews"], flags=flags)
            np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(want.cpu().numpy()), err_msg=f"flags={flags}")
            t = torch.zeros(ops.geom.tiled_count(), device="cuda")
            ops.geom.volume_tiling(dev(g["vol0"]), t, True)
            drv.views(t, b, 0.8, 0, cfg["nviews"], flags=flags, tiled=True)
            x = torch.zeros(ops.vol_shape, device="cuda")
            ops.geom.volume_tiling(t, x, False)
            np.testing.assert_array_equal(bits(x.cpu().numpy()), bits(want.cpu().numpy()), err_msg=f"tiled {flags}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,D", [("cone_wide", 4), ("tbct_slabs", 2)])
def test_solver_with_slabs_equals_reference_loop(name, D, oracle_built):
    """ctr_solver_set_slabs(D) with the reference's backprojection arithmetic:
    three SART + FISTA + FGP-TV iterations (V63/main_recon.cu:344-430) equal
    the reference's D-device loop restated by the oracle, volume bit for bit
    and objectives to 1e-12 (the objective projected by the D-device build's
    row-split projector: V63's one-device projector, for the tetrahedron beam
    its multi-GPU rules); set_slabs(1) then continues with the one-device pass."""
    import gpu_b200
    cfg = SLABS[name]
    o = oracle_built.Oracle(og_desc(cfg))
    split = oracle_built.Oracle(oracle_built.slab_desc(og_desc(cfg), D, -1))
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]]))
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    beta, lam, it = np.float32(0.8), np.float32(0.05), 5
    g = gpu_b200.Geometry(ctr_desc(cfg))
    s = gpu_b200.Solver(g, gpu_b200.F32, beta=float(beta), lambda_tv=float(lam), fgp_iters=it, fista=True,
                        objective=True, use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    s.set_slabs(D)
    s.set_sinogram(dev(b))
    s.set_volume(None)
    objs = s.iterate(3)
    out = torch.zeros(o.vol_shape, device="cuda")
    s.get_volume(out)
    y = np.zeros(o.vol_shape, np.float32)
    xprev = np.zeros_like(y)
    t = np.float32(1.0)
    want = []
    for _ in range(3):
        x = o.fgp(o.sart_pass_slabs(y, b, beta, D), beta * lam, it)
        t_k = (np.float32(1.0) + np.sqrt(np.float32(1.0) + np.float32(4.0) * t * t, dtype=np.float32)) / np.float32(2.0)
        y, xprev = o.fista_momentum(y, xprev, x, t, t_k)
        t = np.float32(t_k)
        fid = o.l2_norm(np.stack([split.forward_view(x, j, 0) for j in range(cfg["nviews"])]), b)
        tv = o.tv_norm(x)
        want.append((tv, fid, fid + 2.0 * float(lam) * tv))
    np.testing.assert_array_equal(bits(out.cpu().numpy()), bits(xprev))
    np.testing.assert_allclose(objs, np.array(want), rtol=1e-12)
    # back to the one-device pass for the next iteration
    s.set_slabs(1)
    s.iterate(1)
    s.get_volume(out)
    x = o.fgp(o.sart_pass_ref(y, b, beta), beta * lam, it)
    t_k = (np.float32(1.0) + np.sqrt(np.float32(1.0) + np.float32(4.0) * t * t, dtype=np.float32)) / np.float32(2.0)
    _, xprev = o.fista_momentum(y, xprev, x, t, t_k)
    np.testing.assert_array_equal(bits(out.cpu().numpy()), bits(xprev))
    s.close()


@pytest.mark.parametrize("name,D", CASES)
def test_row_split_projector(name, D):
    """ctr_geometry_create_slab(desc, D, -1): the whole volume projected as the
    D-device build's row-split projector does (golden, from its kernels)."""
    import gpu_b200
    g = load(name)
    geom = gpu_b200.Geometry(ctr_desc(SLABS[name]), D, -1)
    assert geom.vol_shape == g["vol0"].shape and geom.slab_info() == (1, 0, 0)
    out = torch.zeros((1,) + geom.view_shape, device="cuda")
    j = int(g["view"])
    geom.forward(dev(g["vol0"]), out, j, 1)
    np.testing.assert_array_equal(bits(out[0].cpu().numpy()), bits(g[f"fwd_split_{D}"]))
