"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Bit-exact: Siddon ray sums, the voxel index sequence of every ray (segment
count + FNV hash of the indices), FGP, FISTA momentum, the FDK weight and
backprojection stages.  Floating-point tolerance (stated per test): the
gather backprojector against the scatter adjoint of the oracle's projector
(the same chord lengths summed in another order), the SART pass, the ramp
filter (FP32 convolution against the FP64 kernel), FP64 reductions.
"""
import numpy as np
import pytest

from scan_configs import CONFIG0, NEAR_DETECTOR, NO_ON_PLANE_RAYS, SMALL, STYLES, TBCT, ctr_desc, og_desc_xyz

FP_CASES = dict(SMALL, near_detector=NEAR_DETECTOR, **STYLES, **TBCT)
BP_CASES = dict(SMALL, **STYLES, **TBCT)
# the fan-slice scan has no ray on a voxel plane either (its rows sit at voxel
# centres), nor have the even and the offset tetrahedron-beam scans
NO_ON_PLANE = NO_ON_PLANE_RAYS + ["fan_slices", "tbct", "tbct_odd"]

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def pair(cfg, oracle_built, entry64=False):
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(cfg, entry64))
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    return g, o


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def host(t):
    torch.cuda.synchronize()
    return t.float().cpu().numpy()


@pytest.mark.parametrize("name", sorted(FP_CASES))
def test_forward_bit_exact(name, oracle_built):
    cfg = FP_CASES[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(7)
    vol = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    sino = torch.zeros((cfg["nviews"],) + o.view_shape, device="cuda")
    g.forward(dev(vol), sino)
    out = host(sino)
    for j in range(cfg["nviews"]):
        np.testing.assert_array_equal(bits(out[j]), bits(o.forward_view(vol, j, 0)), err_msg=f"view {j}")


@pytest.mark.parametrize("name", sorted(FP_CASES))
@pytest.mark.parametrize("entry64", [False, True])
def test_traversal_index_sets(name, entry64, oracle_built):
    """Every ray visits the same voxel index sequence as the restated reference."""
    cfg = FP_CASES[name]
    g, o = pair(cfg, oracle_built, entry64)
    vol = np.zeros(o.vol_shape, np.float32)
    P = o.view_shape
    nseg = torch.zeros(P, dtype=torch.int32, device="cuda")
    hsh = torch.zeros(P, dtype=torch.int64, device="cuda")
    ln = torch.zeros(P, dtype=torch.float32, device="cuda")
    dvol = dev(vol)
    for j in range(cfg["nviews"]):
        g.forward_trace(dvol, j, nseg, hsh, ln)
        n_ref, h_ref, l_ref = o.forward_trace(vol, j, entry64)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(nseg.cpu().numpy(), n_ref)
        np.testing.assert_array_equal(hsh.cpu().numpy().view(np.uint64), h_ref)
        np.testing.assert_array_equal(bits(ln.cpu().numpy()), bits(l_ref))


def test_forward_config0_bit_exact(oracle_built):
    """The 128^3 / 128^2 / 180-view scan: a spread of views, bit for bit."""
    g, o = pair(CONFIG0, oracle_built)
    rng = np.random.default_rng(3)
    vol = rng.uniform(0, 0.03, o.vol_shape).astype(np.float32)
    views = [0, 1, 44, 45, 89, 90, 133, 179]
    sino = torch.zeros((180,) + o.view_shape, device="cuda")
    g.forward(dev(vol), sino)
    out = host(sino)
    for j in views:
        np.testing.assert_array_equal(bits(out[j]), bits(o.forward_view(vol, j, 0)), err_msg=f"view {j}")


@pytest.mark.parametrize("name", sorted(BP_CASES))
def test_adjoint_matches_scatter_of_projector(name, oracle_built):
    """Gather adjoint == scatter of the projector's own segments: the same
    chords, FP64 sums in another order, rounded once to float."""
    cfg = BP_CASES[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(11)
    y = rng.standard_normal((cfg["nviews"],) + o.view_shape).astype(np.float32)
    vol = torch.zeros(o.vol_shape, device="cuda")
    g.backproject(dev(y), vol)
    got = host(vol).astype(np.float64)
    ref = o.adjoint(y)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
    # to float rounding, voxel by voxel
    assert np.all(np.abs(got - ref) <= 1.2e-7 * np.abs(ref) + 1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", sorted(BP_CASES))
def test_dot_product(name, oracle_built):
    """<Ax, y> = <x, A^T y> to 1e-6 relative on 16 seeded pairs (x uniform over
    all voxels, y normal over all detector bins)."""
    cfg = BP_CASES[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(5)
    for _ in range(16):
        x = rng.uniform(0, 1, g.vol_shape).astype(np.float32)
        y = rng.standard_normal((cfg["nviews"],) + g.view_shape).astype(np.float32)
        a, b = g.dot_test(dev(x), dev(y))
        assert abs(a - b) <= 1e-6 * max(abs(a), abs(b)), (a, b)
    # and against the oracle's FP64 sums of the same segments
    ref = float(np.sum(o.adjoint(y) * x))
    assert b == pytest.approx(ref, rel=1e-6, abs=1e-9 * np.abs(o.adjoint(y)).sum())


@pytest.mark.parametrize("name", NO_ON_PLANE_RAYS)
def test_masked_adjoint_vs_reference_bp(name, oracle_built):
    """Reference command-0 BP semantics (FOV mask, thresholds) against the
    reference kernel's own alpha formula: equal up to alpha rounding."""
    import gpu_b200
    cfg = SMALL[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(13)
    for j in (0, cfg["nviews"] // 2):
        c = rng.standard_normal(o.view_shape).astype(np.float32)
        vol = torch.zeros(o.vol_shape, device="cuda")
        g.backproject(dev(c[None]), vol, j, 1, flags=gpu_b200.BP_FOV_MASK)
        got = host(vol)
        ref = o.backproject_ref(np.zeros(o.vol_shape, np.float32), c, j, 1.0, 0)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 2e-3 * scale


def test_tbct_has_no_masked_command0(oracle_built):
    """V63's command 0 (CTR_BP_FOV_MASK) is not defined for the tetrahedron
    beam, whose backprojector has no command argument: refused."""
    import gpu_b200
    cfg = TBCT["tbct"]
    g, o = pair(cfg, oracle_built)
    c = torch.zeros((1,) + o.view_shape, device="cuda")
    vol = torch.zeros(o.vol_shape, device="cuda")
    with pytest.raises(gpu_b200.CtrError):
        g.backproject(c, vol, 0, 1, flags=gpu_b200.BP_FOV_MASK)


@pytest.mark.parametrize("name", sorted(BP_CASES))
def test_sart_pass(name, oracle_built):
    """The SART pass equals the restated engine algorithm bit for bit, and the
    reference's own BP (its alpha formula) to alpha rounding (for the
    tetrahedron beam: its backprojection and update)."""
    cfg = BP_CASES[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(17)
    truth = rng.uniform(0, 0.05, o.vol_shape).astype(np.float32)
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    vol = torch.zeros(o.vol_shape, device="cuda")
    g.sart_pass(vol, dev(b), 0.8)
    got = host(vol)
    exact = o.sart_pass_gather(np.zeros_like(truth), b, 0.8)
    np.testing.assert_array_equal(bits(got), bits(exact))
    if name in NO_ON_PLANE:
        ref = o.sart_pass_ref(np.zeros_like(truth), b, 0.8)
        scale = np.abs(ref).max()
        assert np.sqrt(np.mean((got - ref) ** 2)) <= 2e-3 * scale


def test_reference_bp_drops_on_plane_rays(oracle_built):
    """The reference BP evaluates 0/0 for a ray lying exactly on a voxel plane
    and drops it, though its FP traverses it; the engine backprojects the
    FP's own chord.  One-hot correction on the central ray of an odd detector."""
    import gpu_b200
    cfg = SMALL["odd"]
    g, o = pair(cfg, oracle_built)
    c = np.zeros(o.view_shape, np.float32)
    c[cfg["nv"] // 2, cfg["nu"] // 2] = 1.0
    ref = o.backproject_ref(np.zeros(o.vol_shape, np.float32), c, 0, 1.0, 0)
    assert np.count_nonzero(ref) == 0
    vol = torch.zeros(o.vol_shape, device="cuda")
    g.backproject(dev(c[None]), vol, 0, 1, flags=gpu_b200.BP_FOV_MASK)
    got = host(vol)
    n_ref, _, _ = o.forward_trace(np.zeros(o.vol_shape, np.float32), 0)
    assert n_ref[cfg["nv"] // 2, cfg["nu"] // 2] > 0
    chords = o.adjoint_view(c, 0, thresh=True)          # the FP's segments of that ray
    inside = ~o.fov_mask()[None, :, :]
    expected = (chords * inside).astype(np.float32)
    assert expected.sum() > 0
    np.testing.assert_allclose(got, expected, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("name", sorted(SMALL))
def test_fgp_bit_exact(name, oracle_built):
    cfg = SMALL[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(19)
    f = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    for lam, it in ((0.02, 5), (0.3, 20)):
        vol = dev(f)
        g.fgp_tv(vol, lam, it)
        np.testing.assert_array_equal(bits(host(vol)), bits(o.fgp(f, lam, it)))


def test_fista_momentum_bit_exact(oracle_built):
    cfg = SMALL["cube16"]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(23)
    x = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    xp = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    t_prev = 1.0
    t_k = (1.0 + np.sqrt(np.float32(1.0 + 4.0 * t_prev * t_prev), dtype=np.float32)) / np.float32(2.0)
    y, xprev = torch.zeros_like(dev(x)), dev(xp)
    g.fista_momentum(y, xprev, dev(x), np.float32(t_prev), np.float32(t_k))
    ry, rxp = o.fista_momentum(np.zeros_like(x), xp, x, np.float32(t_prev), np.float32(t_k))
    np.testing.assert_array_equal(bits(host(y)), bits(ry))
    np.testing.assert_array_equal(bits(host(xprev)), bits(rxp))


@pytest.mark.parametrize("name", ["cube16", "aniso"])
def test_objective(name, oracle_built):
    cfg = SMALL[name]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(29)
    vol = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    b = rng.uniform(0, 10, (cfg["nviews"],) + o.view_shape).astype(np.float32)
    fid, tv = g.objective(dev(vol), dev(b))
    ax = np.stack([o.forward_view(vol, j, 0) for j in range(cfg["nviews"])])
    assert fid == pytest.approx(o.l2_norm(ax, b), rel=1e-12)
    assert tv == pytest.approx(o.tv_norm(vol), rel=1e-12)


@pytest.mark.parametrize("name", ["cube16", "odd", "aniso"])
def test_fdk(name, oracle_built):
    cfg = SMALL[name]
    g, o = pair(cfg, oracle_built)
    params = np.array([[0, 0, 0, 4, 3, 3.5, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]])
    truth = o.phantom(params)
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    vol = torch.zeros(o.vol_shape, device="cuda")
    g.fdk(dev(b), vol)
    got = host(vol)
    ref = o.fdk(b)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("case", ["cube16", "odd", "aniso", "short_scan"])
def test_fdk_backprojection_bit_exact(case, oracle_built):
    """The FDK backprojection stage alone, on arbitrary filtered views, view by
    view into a non-zero volume: bit-exact against the reference's kernel
    arithmetic.  The full-circle scans take the exact shortcut of the FP64
    factor 360/(us_rate*Nviews) = 1; the short scan (0.5 degree steps over
    6 degrees) takes the FP64 multiply and divide."""
    import gpu_b200
    from oracle import ctoracle
    cfg = dict(SMALL["cube16"] if case == "short_scan" else SMALL[case])
    us = 0.5 if case == "short_scan" else 360.0 / cfg["nviews"]
    g = gpu_b200.Geometry(gpu_b200.make_desc(cfg["nx"], cfg["ny"], cfg["nz"], cfg["vx"], cfg["nu"], cfg["nv"],
                                             cfg["du"], cfg["dso"], cfg["dod"], cfg["nviews"], us_rate=us,
                                             initial_angle=cfg.get("initial_angle", 0.0),
                                             shift_angle=cfg.get("shift_angle", 0.0), offset=cfg.get("offset", 0.0),
                                             m_offset=cfg.get("m_offset", 0)))
    d = og_desc_xyz(cfg)
    d.us_rate = us
    o = ctoracle.Oracle(d)
    rng = np.random.default_rng(23)
    filt = rng.standard_normal((cfg["nviews"],) + o.view_shape).astype(np.float32)
    vol0 = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    vol = dev(vol0)
    half = cfg["nviews"] // 2
    g.fdk_backproject(dev(filt[:half]), vol, 0, half)
    g.fdk_backproject(dev(filt[half:]), vol, half, cfg["nviews"] - half)
    want = vol0
    for j in range(cfg["nviews"]):
        want = o.fdk_bp_view(want, filt[j], j)
    np.testing.assert_array_equal(bits(host(vol)), bits(want))
    assert not np.array_equal(want, vol0)


def test_mixed_precision_forward_exact(oracle_built):
    """BF16/F16 volumes are widened exactly: A(bf16 x) == A(float(bf16 x)) bit for bit."""
    cfg = SMALL["cube16"]
    g, o = pair(cfg, oracle_built)
    rng = np.random.default_rng(31)
    vol = dev(rng.uniform(0, 1, o.vol_shape).astype(np.float32))
    for dt in (torch.bfloat16, torch.float16):
        lo = vol.to(dt)
        s1 = torch.zeros((cfg["nviews"],) + o.view_shape, device="cuda")
        s2 = torch.zeros_like(s1)
        g.forward(lo, s1)
        g.forward(lo.float(), s2)
        np.testing.assert_array_equal(bits(host(s1)), bits(host(s2)))


def test_reference_compatible_entry_points(oracle_built, capfd):
    import gpu_b200
    cfg = SMALL["cube16"]
    gpu_b200.set_default_geometry(ctr_desc(cfg))
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    rng = np.random.default_rng(37)
    vol = rng.uniform(0, 0.05, o.vol_shape).astype(np.float32)
    proj = np.zeros((cfg["nviews"],) + o.view_shape, np.float32)
    gpu_b200.forward_3d_ray_driven_siddon(vol, proj)
    for j in range(cfg["nviews"]):
        np.testing.assert_array_equal(bits(proj[j]), bits(o.forward_view(vol, j, 0)))
    f = vol.copy()
    gpu_b200.fgp_denoise_gpux7_exact(f, 0.01, 5)
    np.testing.assert_array_equal(bits(f), bits(o.fgp(vol, 0.01, 5)))
    assert gpu_b200.tv_norm_gpu(vol) == pytest.approx(o.tv_norm(vol), rel=1e-12)
    noisy = (proj * 1.01).astype(np.float32)
    assert gpu_b200.l2_norm_gpu(proj, noisy) == pytest.approx(o.l2_norm(proj, noisy), rel=1e-12)
    x = np.zeros_like(vol)
    gpu_b200.reconstruction_3d_ray_driven_cbct(x, proj, 0.8)        # the reference's own SART pass
    np.testing.assert_array_equal(bits(x), bits(o.sart_pass_ref(np.zeros_like(vol), proj, 0.8)))
    gpu_b200.check_matched_joint_operator(vol)
    out = capfd.readouterr().out
    assert "The 1st inner product" in out and "The 2nd inner product" in out
    fdk = np.zeros_like(vol)
    gpu_b200.reconstruction_fdk(fdk, proj)
    ref = o.fdk(proj)
    assert np.abs(fdk - ref).max() <= 1e-4 * np.abs(ref).max()
