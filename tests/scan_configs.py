"""Small scan descriptions shared by the tests (sizes in millimetres).

Each entry: nx, ny, nz, nu, nv, nviews, vx, du, dso, dod, and optional
offset, m_offset, initial_angle, shift_angle.  The odd detector sizes put a
detector column and row exactly on the central ray, so axis-parallel rays
exist; the angle steps hit 0, 90, 180 and 270 degrees.
"""

SMALL = {
    "cube16": dict(nx=16, ny=16, nz=16, nu=24, nv=20, nviews=12, vx=1.0, du=1.6, dso=1000.0, dod=-500.0),
    "odd": dict(nx=12, ny=12, nz=12, nu=17, nv=13, nviews=8, vx=1.0, du=1.6, dso=1000.0, dod=-500.0),
    "fine": dict(nx=20, ny=20, nz=20, nu=31, nv=9, nviews=16, vx=0.5, du=0.4, dso=1000.0, dod=-500.0),
    "aniso": dict(nx=18, ny=14, nz=10, nu=27, nv=15, nviews=10, vx=1.0, du=1.6, dso=1000.0, dod=-500.0,
                  offset=0.8, m_offset=1, initial_angle=3.5, shift_angle=1.25),
    "fine_even": dict(nx=20, ny=20, nz=20, nu=30, nv=10, nviews=16, vx=0.5, du=0.4, dso=1000.0, dod=-500.0,
                      initial_angle=1.5),
}

# The volume within 1e-3 mm of the detector plane: alphas inside the volume
# below 1e-6, where the projector keeps the reference's loop test as written
# instead of the single-comparison form.
NEAR_DETECTOR = dict(nx=16, ny=16, nz=16, nu=48, nv=40, nviews=12, vx=1.0, du=0.4, dso=1000.0, dod=-11.3147,
                     initial_angle=7.0)

# Scans with no ray lying exactly on a voxel plane.  On such a ray the
# reference BP evaluates 0/0 and drops the ray while the reference FP keeps it
# (V63/kernel_IterativeRecon_universal.cu:760-765 versus :218-266), so
# comparisons against the reference BP's own arithmetic use these scans.
NO_ON_PLANE_RAYS = ["cube16", "fine_even"]

# the reference's sample configuration, scaled down in resolution only
# (128^3, 1 mm voxels, 128^2 detector at 1.6 mm, 180 views over 360 degrees)
CONFIG0 = dict(nx=128, ny=128, nz=128, nu=128, nv=128, nviews=180, vx=1.0, du=1.6, dso=1000.0, dod=-500.0)


# The reference's other scanner geometries (CT_style 1 and 2), z pitch equal
# to the detector pitch as the reference sets it; odd and even detectors.
STYLES = {
    "fan_slices": dict(nx=16, ny=16, nz=12, nu=24, nv=12, nviews=12, vx=1.0, du=1.2, dso=1000.0, dod=-500.0,
                       ct_style=1),
    "fan_slices_odd": dict(nx=12, ny=12, nz=9, nu=17, nv=9, nviews=8, vx=1.0, du=1.6, dso=1000.0, dod=-500.0,
                           initial_angle=3.5, ct_style=1),
    "parallel": dict(nx=16, ny=16, nz=12, nu=24, nv=12, nviews=12, vx=1.0, du=1.2, dso=1000.0, dod=-500.0,
                     ct_style=2),
    "parallel_odd": dict(nx=12, ny=12, nz=9, nu=17, nv=9, nviews=8, vx=1.0, du=1.6, dso=1000.0, dod=-500.0,
                         initial_angle=3.5, ct_style=2),
}

# The tetrahedron-beam program (TBCT v4.2): n_sources sources stacked along z,
# placed by the reference's automatic distribution, nv detector rows each.
# Magnification 2 as in its sample configuration (DSO = -DOD); adjacent
# sources' bands overlap in the volume.  "tbct_one": a single source at z = 0
# and an odd row count, so the central row's rays lie in a z plane;
# "tbct_odd": odd sizes, detector offset, M_Offset and shift angle.
TBCT = {
    "tbct": dict(nx=16, ny=16, nz=16, nu=32, nv=4, nviews=12, vx=1.0, du=1.2, dso=40.0, dod=-40.0,
                 ct_style=3, n_sources=8),
    "tbct_odd": dict(nx=15, ny=17, nz=13, nu=31, nv=3, nviews=8, vx=1.0, du=1.1, dso=50.0, dod=-30.0,
                     offset=0.7, m_offset=1, shift_angle=3.0, ct_style=3, n_sources=3),
    "tbct_one": dict(nx=16, ny=16, nz=16, nu=33, nv=5, nviews=8, vx=1.0, du=1.2, dso=40.0, dod=-40.0,
                     ct_style=3, n_sources=1),
}


# The multi-GPU build's z split (V63/main_recon.cu:23 Number_of_Devices): nz
# and nv split into each listed slab count.  "cone_wide": a wide cone
# (magnification 2, +-8 degrees), so rays cross slab boundaries and a ray's
# sum is the sum of its slabs' sums; "pitch07": a voxel pitch whose slab
# planes round differently from the whole volume's, and an odd detector whose
# central row's rays lie in a z plane; "fan_edges": fan-slice rows lying
# exactly on slab boundary planes (traced by neither slab); "parallel_slabs":
# the parallel beam.
SLABS = {
    "cube16": dict(SMALL["cube16"], slabs=[2, 4]),
    "cone_wide": dict(nx=16, ny=16, nz=16, nu=24, nv=24, nviews=10, vx=1.0, du=1.0, dso=40.0, dod=-40.0,
                      initial_angle=1.0, slabs=[2, 4]),
    "pitch07": dict(nx=14, ny=14, nz=12, nu=22, nv=15, nviews=8, vx=0.7, du=1.3, dso=1000.0, dod=-500.0,
                    initial_angle=2.0, slabs=[3]),
    "fan_edges": dict(nx=12, ny=12, nz=12, nu=17, nv=9, nviews=8, vx=1.0, du=1.6, dso=1000.0, dod=-500.0,
                      initial_angle=3.5, ct_style=1, slabs=[3]),
    "parallel_slabs": dict(nx=16, ny=16, nz=12, nu=24, nv=12, nviews=12, vx=1.0, du=1.2, dso=1000.0, dod=-500.0,
                           ct_style=2, slabs=[2, 4]),
    # the tetrahedron-beam program's multi-GPU build (its default, T42/main_recon.cu:17)
    "tbct_slabs": dict(TBCT["tbct"], slabs=[2, 4]),
    "tbct_slab3": dict(nx=15, ny=17, nz=12, nu=31, nv=6, nviews=8, vx=1.0, du=1.1, dso=50.0, dod=-30.0, offset=0.7,
                       m_offset=1, shift_angle=3.0, ct_style=3, n_sources=3, slabs=[3]),
}


def og_desc(cfg):
    from oracle.ctoracle import make_desc
    return make_desc(cfg["nx"], cfg["ny"], cfg["nz"], cfg["nu"], cfg["nv"], cfg["nviews"], cfg["vx"], cfg["du"],
                     cfg["dso"], cfg["dod"], initial_angle=cfg.get("initial_angle", 0.0),
                     shift_angle=cfg.get("shift_angle", 0.0), offset=cfg.get("offset", 0.0),
                     m_offset=cfg.get("m_offset", 0), ct_style=cfg.get("ct_style", 0),
                     n_sources=cfg.get("n_sources", 0))


def view_rows(cfg):
    """Detector rows of one view: every source's band for the tetrahedron beam."""
    return cfg["nv"] * (cfg.get("n_sources", 1) if cfg.get("ct_style", 0) == 3 else 1)


def og_desc_xyz(cfg):
    """Oracle description with independent nx, ny, nz."""
    d = og_desc(cfg)
    d.nx, d.ny, d.nz = cfg["nx"], cfg["ny"], cfg["nz"]
    return d


def ctr_desc(cfg, entry64=False, fast_sums=False):
    from gpu_b200.ctrecon import make_desc
    return make_desc(cfg["nx"], cfg["ny"], cfg["nz"], cfg["vx"], cfg["nu"], cfg["nv"], cfg["du"], cfg["dso"],
                     cfg["dod"], cfg["nviews"], initial_angle=cfg.get("initial_angle", 0.0),
                     shift_angle=cfg.get("shift_angle", 0.0), offset=cfg.get("offset", 0.0),
                     m_offset=cfg.get("m_offset", 0), entry64=entry64, ct_style=cfg.get("ct_style", 0),
                     n_sources=cfg.get("n_sources", 0), fast_sums=fast_sums)

# Differentiation scan: 256^3, 360 views, 384^2 detector.  "Config-0 geometry
# scaled by 2" is read as the same physical extents at twice the sampling:
# 0.5 mm voxels (128 mm FOV) and a 204.8 mm detector of 384 pixels.
CONFIG2 = dict(nx=256, ny=256, nz=256, nu=384, nv=384, nviews=360, vx=0.5, du=204.8 / 384, dso=1000.0,
               dod=-500.0)

# Mixed-precision accuracy scan: small enough for the FP64 oracle, an angle
# offset keeps views off the exact axes.
MIXED = dict(nx=64, ny=64, nz=64, nu=96, nv=96, nviews=90, vx=2.0, du=3.2, dso=1000.0, dod=-500.0,
             initial_angle=1.0)

# The same field of view at half the sampling, for the FP64 oracle's
# FISTA-step test on the CPU.
FISTA32 = dict(nx=32, ny=32, nz=32, nu=48, nv=48, nviews=90, vx=4.0, du=6.4, dso=1000.0, dod=-500.0,
               initial_angle=1.0)
