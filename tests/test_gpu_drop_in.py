"""The drop-in from C++: tests/c/drop_in_main.cpp is the reference's FISTA
driver loop (V63/main_recon.cu:286-430) written against the library's
reference-compatible host functions, compiled with g++ against
include/ctrecon.h and linked to the in-tree libctrecon.so.  Its reconstruction
must equal the reference's call sequence restated by the oracle bit for bit,
and its printed objectives the oracle's: for the one-device build, and for
the stock 4-device build (Number_of_Devices 4, whose SART pass is the z-slab
sequence of V63/host_IterativeRecon_CBCT_multiGPU.c) on a wide-cone scan
whose rays cross the slab planes."""
import os
import subprocess

import numpy as np
import pytest

from scan_configs import SLABS, SMALL, og_desc_xyz

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


# the driver takes no initial angle (the reference's initialAngle is 0 in the stock file)
@pytest.mark.parametrize("cfg,devices", [(SMALL["cube16"], 1), (dict(SLABS["cone_wide"], initial_angle=0.0), 4)],
                         ids=["one_device", "four_devices"])
def test_cpp_driver_equals_reference_sequence(cfg, devices, tmp_path, oracle_built):
    exe = tmp_path / "drop_in_main"
    lib = os.path.join(ROOT, "gpu_b200")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "drop_in_main.cpp"), "-o", str(exe), "-L", lib, "-lctrecon",
                    f"-Wl,-rpath,{lib}"], check=True)
    o = oracle_built.Oracle(og_desc_xyz(cfg))
    truth = o.phantom(np.array([[0, 0, 0, 5, 4, 3, 0.3, 0.2, 0.1, 0.02], [1.5, -1, 0.5, 2, 2, 2, 0, 0, 0, 0.03]]))
    b = np.stack([o.forward_view(truth, j, 0) for j in range(cfg["nviews"])])
    b.tofile(tmp_path / "sino.raw")
    beta, lam, fgp_iters, iters = np.float32(0.8), np.float32(0.05), 5, 3
    args = [cfg["nx"], cfg["ny"], cfg["nz"], cfg["vx"], cfg["nu"], cfg["nv"], cfg["du"], cfg["dso"], cfg["dod"],
            cfg["nviews"], iters, float(beta), float(lam), fgp_iters, tmp_path / "sino.raw", tmp_path / "vol.raw",
            devices]
    run = subprocess.run([str(exe)] + [str(a) for a in args], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    got = np.fromfile(tmp_path / "vol.raw", np.float32).reshape(o.vol_shape)
    objs = np.array([[float(v) for v in line.split()[1:]] for line in run.stdout.strip().splitlines()])

    # the reference's loop, restated: its SART pass, FGP x7, FISTA step, objective
    y = np.zeros(o.vol_shape, np.float32)
    xprev = np.zeros_like(y)
    t = np.float32(1.0)
    want_objs = []
    for _ in range(iters):
        sart = o.sart_pass_ref(y, b, beta) if devices == 1 else o.sart_pass_slabs(y, b, beta, devices)
        x = o.fgp(sart, beta * lam, fgp_iters)
        t_k = (np.float32(1.0) + np.sqrt(np.float32(1.0) + np.float32(4.0) * t * t, dtype=np.float32)) / np.float32(2.0)
        y, xprev = o.fista_momentum(y, xprev, x, t, t_k)
        t = np.float32(t_k)
        ax = np.stack([o.forward_view(x, j, 0) for j in range(cfg["nviews"])])
        fid, tv = o.l2_norm(ax, b), o.tv_norm(x)
        want_objs.append((tv, fid, fid + 2.0 * float(lam) * tv))
    np.testing.assert_array_equal(got.view(np.uint32), xprev.view(np.uint32))
    np.testing.assert_allclose(objs, np.array(want_objs), rtol=1e-12)
    assert objs[-1, 1] < objs[0, 1]
