"""The refinement solver (``refine=True``): FP32 FISTA state, 16-bit copies
for the projectors and a 16-bit correction volume d accumulated per SART
pass against the FP32 residual b - A y_k.

Its call sequence is restated here from oracle functions (the engine's
Siddon sums, chord lengths and gather update, float32 numpy arithmetic) and
the GPU result must equal it bit for bit: with FP32 storage including FGP-TV
(whose duals the restatement keeps in float), with FP16 storage without FGP.
The batch and a checkpoint resume must give the single solver's bits."""
import numpy as np
import pytest

from scan_configs import SMALL, TBCT, ctr_desc, og_desc_xyz

SCANS = dict(SMALL, **TBCT)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

PHANTOM = np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]])
F = np.float32


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def store(x, dtype):
    return x.astype(np.float16).astype(np.float32) if dtype == "f16" else x.astype(np.float32)


def refine_restated(o, b, beta, lam_tv, fgp_iters, n_iter, dtype, fista=True, d32=False):
    """The refinement iteration in float32 from oracle primitives; returns the
    FP32 x_k and the fidelity of each iteration's 16-bit copy.  d32: the
    correction volume kept in FP32 (refine=2)."""
    dstore = (lambda x: x.astype(np.float32)) if d32 else (lambda x: store(x, dtype))
    nv = b.shape[0]
    xk = np.zeros(o.vol_shape, F)
    xm = np.zeros_like(xk)
    ax = np.zeros(b.shape, F)          # A x~_(k-1) per ray, from the previous pass
    t, gm = F(1.0), F(0.0)
    fids = []
    for _ in range(n_iter):
        xc = store(xk, dtype)          # the projectors' copy of x_k
        # d starts at the copies' rounding of y_k = (1+g) x_k - g x_(k-1)
        d0 = dstore((F(1.0) + gm) * (xk - xc) - gm * (xm - store(xm, dtype)))
        d = d0.copy()
        for j in range(nv):
            sx = o.forward_view(xc, j, 0)                    # A x~_k, zero below vz*1e-6
            sd = o.forward_view(d, j, 0)                     # A d (its rays above the threshold)
            _, _, ln = o.forward_trace(xc, j)
            ay = (F(1.0) + gm) * sx - gm * ax[j]
            zero = ln < F(o.desc.vz) * F(1e-6)
            c = np.where(zero, F(0.0), ((b[j] - ay) - sd) / np.where(zero, F(1.0), ln)).astype(F)
            ax[j] = sx
            d = dstore(o.backproject_gather(d, c, j, beta))
        fids.append(float(np.sum(((ax - b).astype(F) ** 2).astype(np.float64))))
        z = ((F(1.0) + gm) * xk - gm * xm + (d - d0)).astype(F)
        xs = o.fgp(z, F(beta) * F(lam_tv), fgp_iters) if lam_tv > 0 else z
        xm, xk = xk, xs.astype(F)
        t_k = (F(1.0) + np.sqrt(F(1.0) + F(4.0) * t * t, dtype=F)) / F(2.0)
        if fista:
            gm = F((t - F(1.0)) / t_k)
            t = F(t_k)
    return xk, fids


def problem(oracle_mod, name):
    cfg = SCANS[name]
    o = oracle_mod.Oracle(og_desc_xyz(cfg))
    b = np.stack([o.forward_view(o.phantom(PHANTOM), j, 0) for j in range(cfg["nviews"])])
    return cfg, o, b


@pytest.mark.parametrize("name", ["cube16", "aniso", "tbct"])
@pytest.mark.parametrize("dtype,lam,refine", [("f32", 0.05, 1), ("f16", 0.0, 1), ("f16", 0.0, 2)])
def test_refine_matches_restatement(name, dtype, lam, refine, oracle_built):
    """refine=2: the correction volume in FP32 while the copies are FP16."""
    import gpu_b200
    cfg, o, b = problem(oracle_built, name)
    beta, fgp_iters, n = 0.3, 4, 3
    vdt, tdt = {"f32": (gpu_b200.F32, torch.float32), "f16": (gpu_b200.F16, torch.float16)}[dtype]
    g = gpu_b200.Geometry(ctr_desc(cfg))
    s = gpu_b200.Solver(g, vdt, beta=beta, lambda_tv=lam, fgp_iters=fgp_iters, fista=True, objective=True,
                        refine=refine)
    s.set_sinogram(torch.from_numpy(b).cuda().to(tdt))
    s.set_volume(None)
    objs = s.iterate(n)
    got = torch.zeros(o.vol_shape, device="cuda")
    s.get_volume_f32(got)
    bq = store(b, dtype)
    want, fids = refine_restated(o, bq, beta, lam, fgp_iters, n + 1, dtype, d32=refine == 2)
    # n + 1 restated passes: the last one's fidelity is the objective of x_n
    want_n, _ = refine_restated(o, bq, beta, lam, fgp_iters, n, dtype, d32=refine == 2)
    np.testing.assert_array_equal(bits(got.cpu().numpy()), bits(want_n))
    np.testing.assert_allclose(objs[:, 1], fids[1:], rtol=1e-12)
    copy = torch.zeros(o.vol_shape, device="cuda", dtype=tdt)
    s.get_volume(copy)
    np.testing.assert_array_equal(bits(copy.float().cpu().numpy()), bits(store(want_n, dtype)))


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("dtype", ["f16", "bf16_sr", "bf16_d32"])
def test_refine_batch_equals_single(dtype, persistent, oracle_built):
    """bf16_d32: BF16 copies with the FP32 correction (refine=2)."""
    import gpu_b200
    vdt, tdt = {"f16": (gpu_b200.F16, torch.float16), "bf16_sr": (gpu_b200.BF16, torch.bfloat16),
                "bf16_d32": (gpu_b200.BF16, torch.bfloat16)}[dtype]
    flags = gpu_b200.SART_STOCHASTIC_ROUND if dtype.endswith("_sr") else 0
    kw = dict(beta=0.3, lambda_tv=0.05, fgp_iters=4, fista=True, objective=True, sart_flags=flags,
              refine=2 if dtype.endswith("_d32") else 1)
    data = [problem(oracle_built, n) for n in ["cube16", "odd", "aniso", "tbct"]]
    geoms = [gpu_b200.Geometry(ctr_desc(cfg)) for cfg, _, _ in data]
    batch = gpu_b200.Batch(geoms, vdt, **kw)
    if persistent:
        batch.set_persistent(True)
    sinos = [torch.from_numpy(b).cuda().to(tdt) for _, _, b in data]
    for i, sb in enumerate(sinos):
        batch.set_sinogram(i, sb)
    batch.reset()
    objs = np.concatenate([batch.iterate(2), batch.iterate(1)], axis=1)
    for i, (cfg, o, _) in enumerate(data):
        s = gpu_b200.Solver(gpu_b200.Geometry(ctr_desc(cfg)), vdt, **kw)
        s.set_sinogram(sinos[i])
        s.set_volume(None)
        ref_obj = s.iterate(3)
        want = torch.zeros(o.vol_shape, device="cuda", dtype=tdt)
        got = torch.zeros_like(want)
        s.get_volume(want)
        batch.get_volume(i, got)
        np.testing.assert_array_equal(bits(got.float().cpu().numpy()), bits(want.float().cpu().numpy()))
        np.testing.assert_array_equal(objs[i], ref_obj)


def test_refine_checkpoint_resume(oracle_built, tmp_path):
    import gpu_b200
    cfg, o, b = problem(oracle_built, "aniso")
    kw = dict(beta=0.3, lambda_tv=0.05, fgp_iters=4, fista=True, objective=True, refine=True)
    sino = torch.from_numpy(b).cuda().half()
    g = gpu_b200.Geometry(ctr_desc(cfg))
    a = gpu_b200.Solver(g, gpu_b200.F16, **kw)
    a.set_sinogram(sino)
    a.set_volume(None)
    a.iterate(2)
    a.save(tmp_path / "ck.bin")
    full = a.iterate(2)
    b2 = gpu_b200.Solver(gpu_b200.Geometry(ctr_desc(cfg)), gpu_b200.F16, **kw)
    b2.set_sinogram(sino)
    b2.load(tmp_path / "ck.bin")
    resumed = b2.iterate(2)
    x1, x2 = torch.zeros(o.vol_shape, device="cuda"), torch.zeros(o.vol_shape, device="cuda")
    a.get_volume_f32(x1)
    b2.get_volume_f32(x2)
    np.testing.assert_array_equal(bits(x1.cpu().numpy()), bits(x2.cpu().numpy()))
    np.testing.assert_array_equal(full, resumed)
    plain = gpu_b200.Solver(gpu_b200.Geometry(ctr_desc(cfg)), gpu_b200.F16, beta=0.3)
    with pytest.raises(gpu_b200.CtrError):
        plain.load(tmp_path / "ck.bin")     # written by a refinement solver


def test_refine_rejects_slabs(oracle_built):
    import gpu_b200
    cfg = SCANS["cube16"]
    s = gpu_b200.Solver(gpu_b200.Geometry(ctr_desc(cfg)), gpu_b200.F16, beta=0.3, refine=True)
    with pytest.raises(gpu_b200.CtrError):
        s.set_slabs(2)
