"""Pin the C restatement (oracle/ct_oracle.c) to the reference.

The golden fixtures were produced by the reference's own kernel sources
compiled for the CPU (tests/golden/make_golden.py), for the cone beam, the
reference's fan-slice and parallel-beam geometries (CT_style 1, 2) and its
tetrahedron-beam program.  The restatement must reproduce them bit for bit:
Siddon FP (command 0 and the SART correction), the voxel-driven BP (command
0 and the SART update), a whole SART pass, FGP, the TV and L2 norms, and the
FDK weight / ramp / backprojection (the tetrahedron beam: FP, its
backprojection + update and its SART pass).
"""
import os

import numpy as np
import pytest

from scan_configs import SMALL, STYLES, TBCT, og_desc_xyz

CASES = dict(SMALL, **STYLES, **TBCT)

HERE = os.path.dirname(os.path.abspath(__file__))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))


# FGP and the norms are the cone-beam program's (the tetrahedron-beam program
# shares them); FDK exists for the cone beam (CT_style 0) only.
FGP_CASES = sorted(n for n in CASES if CASES[n].get("ct_style", 0) != 3)
FDK_CASES = sorted(n for n in CASES if not CASES[n].get("ct_style", 0))


def _case(name, oracle_built):
    cfg = CASES[name]
    return name, cfg, oracle_built.Oracle(og_desc_xyz(cfg)), load(name)


@pytest.fixture(params=sorted(CASES))
def case(request, oracle_built):
    return _case(request.param, oracle_built)


def test_forward_bit_exact(case):
    _, cfg, o, g = case
    for j in range(cfg["nviews"]):
        np.testing.assert_array_equal(bits(o.forward_view(g["vol"], j, 0)), bits(g["fp0"][j]))
        np.testing.assert_array_equal(bits(o.forward_view(g["vol"], j, 1, g["b"][j])), bits(g["fp1"][j]))


def test_backproject_bit_exact(case):
    _, cfg, o, g = case
    for a, j in enumerate(g["bp_views"]):
        np.testing.assert_array_equal(bits(o.backproject_ref(g["vol"], g["corr"][a], int(j), 0.8, 1)), bits(g["bp1"][a]))
        if cfg.get("ct_style", 0) == 3:
            continue   # the tetrahedron-beam backprojector has no command argument
        z = np.zeros_like(g["vol"])
        np.testing.assert_array_equal(bits(o.backproject_ref(z, g["corr"][a], int(j), 1.0, 0)), bits(g["bp0"][a]))


def test_sart_pass_bit_exact(case):
    _, _, o, g = case
    out = o.sart_pass_ref(np.zeros_like(g["vol"]), g["b"], 0.8)
    np.testing.assert_array_equal(bits(out), bits(g["sart"]))


@pytest.mark.parametrize("name", FGP_CASES)
def test_fgp_and_norms_bit_exact(name, oracle_built):
    _, cfg, o, g = _case(name, oracle_built)
    np.testing.assert_array_equal(bits(o.fgp(g["vol"], float(g["fgp_lambda"]), int(g["fgp_iters"]))), bits(g["fgp"]))
    assert o.tv_norm(g["vol"]) == float(g["tv"])
    assert o.l2_norm(g["fp0"], g["b"]) == float(g["l2"])


@pytest.mark.parametrize("name", FDK_CASES)
def test_fdk_stages(name, oracle_built):
    _, cfg, o, g = _case(name, oracle_built)
    np.testing.assert_array_equal(bits(o.fdk_weight(g["b"])), bits(g["fdkw"]))
    ramp = o.ramp_filter(g["fdkw"][:2])
    # the reference filters with a double-precision FFT; the restatement convolves
    # with the exact spatial kernel in double: equal after rounding to float,
    # up to the last bit of a few values
    scale = np.abs(g["ramp"]).max()
    assert np.abs(ramp - g["ramp"]).max() <= 2e-6 * scale
    fdkbp = np.zeros_like(g["vol"])
    for j in range(min(cfg["nviews"], 4)):
        fdkbp = o.fdk_bp_view(fdkbp, g["ramp"][0] if j % 2 == 0 else g["ramp"][1], j)
    np.testing.assert_array_equal(bits(fdkbp), bits(g["fdkbp"]))


@pytest.mark.parametrize("name", ["odd", "fan_slices_odd", "parallel_odd", "tbct_odd"])
def test_against_reference_build_directly(name, oracle_built):
    """When the reference checkout was compiled here, compare on fresh seeds too."""
    cfg = CASES[name]
    if not os.path.exists(oracle_built.REF_SO_STYLE[cfg.get("ct_style", 0)]):
        pytest.skip("oracle/_ref not built (no reference checkout)")
    d = og_desc_xyz(cfg)
    o, r = oracle_built.Oracle(d), oracle_built.RefOracle(d)
    rng = np.random.default_rng(99)
    vol = rng.uniform(0, 1, o.vol_shape).astype(np.float32)
    for j in range(cfg["nviews"]):
        assert o.trig(j) == r.trig(j)
        np.testing.assert_array_equal(bits(o.forward_view(vol, j, 0)), bits(r.forward_view(vol, j, 0)))
        c = rng.standard_normal(o.view_shape).astype(np.float32)
        np.testing.assert_array_equal(bits(o.backproject_ref(vol, c, j, 0.5, 1)), bits(r.backproject_view(vol, c, j, 0.5, 1)))
