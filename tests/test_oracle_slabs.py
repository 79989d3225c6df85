"""Pin the oracle's z-slab SART (the reference's multi-GPU build) to the reference.

The fixtures (tests/golden/make_golden_slabs.py) come from the reference's
multi-GPU kernels (V63/kernel_IterativeRecon_universal_multiGPU.cu) run on
the CPU with its host sequence (V63/host_IterativeRecon_CBCT_multiGPU.c),
the devices a loop over the slabs, and from the tetrahedron-beam program's
own multi-GPU build (T42/voxel/*_multiGPU.*).  The restatement must reproduce, bit for
bit, each slab's partial ray sums, the ordered combination into the SART
correction, the slab backprojections (commands 0 and 1) and whole passes.
Where oracle/_ref is built, the same comparisons also run live on fresh
inputs, and the reference's row-split forward projection is checked against
the oracle's (slab -1) and, for V63, against its one-device projection (the
reason the one-device projector serves V63's D-device
Forward_3D_ray_driven_siddon; T42's multi-GPU projectors use V63's
traversal rules instead of its own).
"""
import os

import numpy as np
import pytest

from scan_configs import SLABS, og_desc

HERE = os.path.dirname(os.path.abspath(__file__))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"slabs_{name}.npz")))


CASES = [(name, D) for name, cfg in SLABS.items() for D in cfg["slabs"]]


def slab_oracles(oracle_built, cfg, D):
    d = og_desc(cfg)
    return [oracle_built.Oracle(oracle_built.slab_desc(d, D, s)) for s in range(D)]


@pytest.mark.parametrize("name,D", CASES)
def test_pieces_equal_reference_golden(name, D, oracle_built):
    cfg = SLABS[name]
    g = load(name)
    j = int(g["view"])
    zs = cfg["nz"] // D
    os_ = slab_oracles(oracle_built, cfg, D)
    w, ln = zip(*[o.forward_partial(g["vol0"][zs * s:zs * (s + 1)], j) for s, o in enumerate(os_)])
    np.testing.assert_array_equal(bits(np.stack(w)), bits(g[f"w_{D}"]))
    np.testing.assert_array_equal(bits(np.stack(ln)), bits(g[f"l_{D}"]))
    corr = os_[0].combine_partials(np.stack(w), np.stack(ln), g["b"][j])
    np.testing.assert_array_equal(bits(corr), bits(g[f"corr_{D}"]))
    bp1 = np.concatenate([o.backproject_ref(g["vol0"][zs * s:zs * (s + 1)], corr, j, 0.8, 1)
                          for s, o in enumerate(os_)])
    np.testing.assert_array_equal(bits(bp1), bits(g[f"bp1_{D}"]))
    bp0 = np.concatenate([o.backproject_ref(np.zeros((zs, cfg["ny"], cfg["nx"]), np.float32), corr, j, 1.0, 0)
                          for o in os_])
    np.testing.assert_array_equal(bits(bp0), bits(g[f"bp0_{D}"]))


@pytest.mark.parametrize("name,D", CASES)
def test_pass_equals_reference_golden(name, D, oracle_built):
    cfg = SLABS[name]
    g = load(name)
    o = oracle_built.Oracle(og_desc(cfg))
    got = o.sart_pass_slabs(g["vol0"], g["b"], 0.8, D)
    np.testing.assert_array_equal(bits(got), bits(g[f"sart_{D}"]))


def test_slab_pass_is_not_the_one_device_pass(oracle_built):
    """The split changes the numbers: a wide cone's rays cross the slab planes
    at z = +-4 (not the one at z = 0, the source's height), the 0.7 mm slabs'
    planes round differently, and fan-slice rows on a slab plane are traced by
    neither slab."""
    for name, D in (("cone_wide", 4), ("pitch07", 3), ("fan_edges", 3), ("tbct_slabs", 4)):
        cfg = SLABS[name]
        g = load(name)
        o = oracle_built.Oracle(og_desc(cfg))
        one = o.sart_pass_ref(g["vol0"], g["b"], 0.8)
        assert np.count_nonzero(one != g[f"sart_{D}"]) > 0, name


def test_slab_geometry_rejects_uneven_splits(oracle_built):
    cfg = SLABS["pitch07"]                 # nz 12, nv 15
    d = og_desc(cfg)
    for D in (2, 4, 5):                    # 15 rows or 12 slices do not split
        with pytest.raises(ValueError):
            oracle_built.Oracle(oracle_built.slab_desc(d, D, 0))
    tb = og_desc(dict(nx=16, ny=16, nz=16, nu=32, nv=4, nviews=4, vx=1.0, du=1.2, dso=40.0, dod=-40.0,
                      ct_style=3, n_sources=2))
    for D in (3, 8):                       # 16 slices / 4 rows per band do not split
        with pytest.raises(ValueError):
            oracle_built.Oracle(oracle_built.slab_desc(tb, D, 0))


@pytest.mark.parametrize("name,D", CASES)
def test_row_split_forward_equals_reference_golden(name, D, oracle_built):
    """The D-device build's whole-view projector (slab -1: V63's traversal
    rules, which T42's multi-GPU build also uses) against its kernels' output."""
    g = load(name)
    o = oracle_built.Oracle(oracle_built.slab_desc(og_desc(SLABS[name]), D, -1))
    np.testing.assert_array_equal(bits(o.forward_view(g["vol0"], int(g["view"]), 0)), bits(g[f"fwd_split_{D}"]))


def _ref_or_skip(oracle_built, d, multi=False):
    try:
        return oracle_built.RefOracle(d, multi=multi)
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built (needs the reference checkout)")


@pytest.mark.parametrize("name,D", CASES)
def test_live_against_reference_kernels(name, D, oracle_built):
    """Fresh seeded inputs: the whole pass and the row-split forward, against
    the reference's kernels run now."""
    cfg = SLABS[name]
    d = og_desc(cfg)
    ref = _ref_or_skip(oracle_built, d, multi=True)   # the multi-GPU kernels (T42's own for its scans)
    one = _ref_or_skip(oracle_built, d)
    o = oracle_built.Oracle(d)
    rng = np.random.default_rng(77 + D)
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]]))
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    vol = rng.uniform(0, 0.02, o.vol_shape).astype(np.float32)
    vol[rng.uniform(size=vol.shape) < 0.05] = -0.0
    np.testing.assert_array_equal(bits(o.sart_pass_slabs(vol, b, 0.8, D)), bits(ref.sart_slabs(vol, b, 0.8, D)))
    split = oracle_built.Oracle(oracle_built.slab_desc(d, D, -1))
    for j in (0, cfg["nviews"] - 1):
        want = ref.forward_view_split(truth, D, j)
        np.testing.assert_array_equal(bits(split.forward_view(truth, j, 0)), bits(want))
        if cfg.get("ct_style", 0) != 3:   # V63's row split is its one-device projector
            np.testing.assert_array_equal(bits(want), bits(one.forward_view(truth, j, 0)))
