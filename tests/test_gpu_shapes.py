"""Launch shapes of the SART projectors and their tuner: every forward
projector shape and every backprojector shape (the fixed-shape kernel and
the column walks), on the linear and on the 8x8-tiled volume layout, gives
bit-identical projections and SART passes."""
import numpy as np
import pytest

from scan_configs import SMALL, STYLES, TBCT, ctr_desc, og_desc_xyz

CASES = dict(SMALL, **STYLES, **TBCT)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def bits(t):
    return t.float().cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("name", ["cube16", "odd", "aniso", "fine_even", "fan_slices_odd", "parallel", "tbct",
                                  "tbct_odd"])
@pytest.mark.parametrize("dtype", ["f32", "bf16_sr"])
def test_every_shape_gives_the_same_result(name, dtype, oracle_built):
    import gpu_b200
    cfg = CASES[name]
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]]))
    b = torch.from_numpy(np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])).cuda()
    vdt, tdt = (gpu_b200.F32, torch.float32) if dtype == "f32" else (gpu_b200.BF16, torch.bfloat16)
    flags = gpu_b200.SART_STOCHASTIC_ROUND if dtype.endswith("_sr") else 0
    g = gpu_b200.Geometry(ctr_desc(cfg))
    x0 = torch.from_numpy(truth).cuda().to(tdt)
    ref_fp = ref_sart = None
    for fs in range(g.FP_SHAPES):
        for bs in range(-1, g.BP_SHAPES):
            g.set_shapes(fs, bs)
            assert g.shapes() == (fs, bs)
            fp = torch.zeros_like(b)
            g.forward(x0, fp)
            for tiled in (0, gpu_b200.SART_TILED):
                x = torch.zeros(g.vol_shape, device="cuda", dtype=tdt)
                g.sart_pass(x, b, 0.8, flags=flags | tiled, seed=7)
                g.sart_pass(x, b, 0.8, flags=flags | tiled, seed=8)
                if ref_fp is None:
                    ref_fp, ref_sart = bits(fp), bits(x)
                    assert np.any(ref_sart != 0)
                else:
                    np.testing.assert_array_equal(bits(fp), ref_fp, err_msg=f"fp shape {fs}")
                    np.testing.assert_array_equal(bits(x), ref_sart, err_msg=f"shapes {fs} {bs} tiled {tiled}")


def test_autotune_picks_a_valid_shape():
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(SMALL["fine"]))
    r = g.autotune(gpu_b200.F16, n_views=3)
    assert 0 <= r["fp_shape"] < g.FP_SHAPES and -1 <= r["bp_shape"] < g.BP_SHAPES
    assert all(t > 0 for t in r["fp_ms"]) and all(t > 0 for t in r["bp_ms"].values())
    assert r["fp_ms"][r["fp_shape"]] == min(r["fp_ms"])
    assert r["bp_ms"][r["bp_shape"]] == min(r["bp_ms"].values())
    with pytest.raises(gpu_b200.CtrError):
        g.set_shapes(g.FP_SHAPES, 0)
    with pytest.raises(gpu_b200.CtrError):
        g.set_shapes(0, -2)
