"""FDK's frame.  The reference's FDK backprojects in the +theta frame
(V63/FDK/kernel_FDK.cu:33-34, V63/host_FDK.cpp:37) while its projectors use
-theta, so ``ctr_fdk`` (the reference's output) is the projector frame's
volume with x and y exchanged; ``ctr_fdk_projector_frame`` returns it in the
projectors' frame.  Checked by reconstruction quality: FDK of the forward
projection of a phantom, in the projector frame, against the phantom."""
import numpy as np
import pytest

from scan_configs import ctr_desc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CFG = dict(nx=64, ny=64, nz=64, nu=128, nv=96, nviews=180, vx=2.0, du=3.2, dso=1000.0, dod=-500.0)
PHANTOM = np.array([[20, -10, 5, 15, 8, 10, 0.3, 0.0, 0.0, 0.02], [-15, 25, -10, 6, 6, 12, 0, 0, 0, 0.03],
                    [0, 0, 0, 40, 30, 30, 0, 0, 0, 0.01]])
# RMSE of FDK(FP(phantom)) against the phantom, relative to its maximum, for
# this 180-view cone beam (the oracle's FDK gives 1.24e-2 in the projector
# frame and 5.6e-2 without the exchange)
LIMIT = 1.5e-2


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_fdk_projector_frame_reconstructs_the_phantom():
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(CFG))
    truth = torch.zeros(g.vol_shape, device="cuda")
    g.phantom_voxelize(PHANTOM, truth)
    sino = torch.zeros((CFG["nviews"],) + g.view_shape, device="cuda")
    g.forward(truth, sino)
    ref_frame = g.fdk(sino, torch.zeros_like(truth))
    proj_frame = g.fdk_projector_frame(sino, torch.zeros_like(truth))
    # the same numbers, x and y exchanged
    assert torch.equal(proj_frame, ref_frame.transpose(1, 2).contiguous())
    mu = float(truth.max())
    rmse = float(torch.sqrt(torch.mean((proj_frame - truth) ** 2))) / mu
    rmse_raw = float(torch.sqrt(torch.mean((ref_frame - truth) ** 2))) / mu
    print(f"FDK RMSE against the phantom: projector frame {rmse:.3e}, reference frame {rmse_raw:.3e} of max")
    assert rmse <= LIMIT
    assert rmse_raw > 3 * rmse


def test_fdk_projector_frame_accumulates_and_refuses_offsets():
    import gpu_b200
    g = gpu_b200.Geometry(ctr_desc(CFG))
    sino = torch.rand((CFG["nviews"],) + g.view_shape, device="cuda")
    base = torch.rand(g.vol_shape, device="cuda")
    once = g.fdk_projector_frame(sino, torch.zeros_like(base))
    acc = g.fdk_projector_frame(sino, base.clone())
    # the views are added to the estimate one by one, so the sums round differently
    torch.testing.assert_close(acc, base + once, rtol=1e-4, atol=1e-4 * float(once.abs().max()))
    off = gpu_b200.Geometry(ctr_desc(dict(CFG, offset=0.8)))
    with pytest.raises(gpu_b200.CtrError):
        off.fdk_projector_frame(sino, torch.zeros_like(base))
