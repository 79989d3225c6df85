"""The reference driver's file formats (V63/main_recon.cu:197-266, 434-477):
file names formatted like the reference's sprintf calls, raw round trips, the
per-view reader with the reference's angle rule and row offset.  CPU only."""
import numpy as np
import pytest


def test_view_filenames_follow_the_reference_rule():
    import gpu_b200.ctrecon as ct
    assert ct.view_filename(0, 1.0, 0.0) == "View_0.00.dat"
    assert ct.view_filename(45, 0.3515625, 0.0) == "View_%.02f.dat" % np.float32(45 * np.float32(0.3515625))
    assert ct.view_filename(3, 1.0, -10.0) == "View_353.00.dat"          # negative angle + 360
    # tomosynthesis: the second half starts at 180 degrees
    assert ct.view_filename(6, 2.0, 0.0, tomo=1, n_views=10) == "View_182.00.dat"


def test_recon_and_objective_names():
    import gpu_b200.ctrecon as ct
    n = ct.recon_filename("Ellipsoid", 1024, 1024, 256, 100.0, 1, 0.0, 0.0, 0.0, 0.0, 32.0)
    assert n == "Ellipsoid_1024_1024_256_100um_new_view_1_(0,0)_TV_0.00_L1_0.00_Lip_32.00.recon"
    n = ct.recon_filename("Ellipsoid", 512, 512, 512, 500.0, 1024, 0.0, 359.6, 2e-4, 0.0, 2.5, iteration=6)
    assert n == "Ellipsoid_512_512_512_500um_iterative_6_view_1024_(0,360)_TV_0.00_L1_0.00_Lip_2.50.recon"
    n = ct.objective_filename("Ellipsoid", 1024, 0.0, 359.6, 0.01, 32.0)
    assert n == "object_func_Ellipsoid_view_1024_(0,360)_TV_0.01_Lip_32.00.bin"


def test_views_round_trip_with_row_offset(tmp_path):
    import gpu_b200.ctrecon as ct
    rng = np.random.default_rng(0)
    proj = rng.standard_normal((5, 12, 7)).astype(np.float32)
    ct.write_views(tmp_path, proj, 1.5, 2.0)
    assert (tmp_path / "View_3.50.dat").exists()
    back = ct.read_views(tmp_path, 7, 12, 5, 1.5, 2.0)
    np.testing.assert_array_equal(back, proj)
    part = ct.read_views(tmp_path, 7, 8, 5, 1.5, 2.0, row_offset=4)
    np.testing.assert_array_equal(part, proj[:, 4:, :])


def test_raw_volume_and_objective_files(tmp_path):
    import gpu_b200.ctrecon as ct
    vol = np.arange(4 * 5 * 6, dtype=np.float32).reshape(4, 5, 6)
    ct.write_raw(tmp_path / "v.recon", vol)
    np.testing.assert_array_equal(ct.read_raw(tmp_path / "v.recon", vol.shape), vol)
    obj = np.array([[1.5, 2.5, 3.5], [4.0, 5.0, 6.0]])
    ct.write_raw(tmp_path / "o.bin", obj)
    assert (tmp_path / "o.bin").stat().st_size == 6 * 8
    with pytest.raises(ct.CtrError):
        ct.read_raw(tmp_path / "v.recon", (5, 5, 6))
    with pytest.raises(ct.CtrError):
        ct.read_views(tmp_path / "missing", 7, 12, 5, 1.5)
