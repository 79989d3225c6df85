"""ctypes binding of ``libctrecon.so`` (``include/ctrecon.h``).

The library is the product; this module only marshals arguments.  Device
buffers are torch CUDA tensors (their ``data_ptr()``), streams are torch
streams (``cuda_stream``); host buffers for the reference-compatible entry
points are numpy arrays.  Every call checks the returned ``ctr_status`` and
raises :class:`CtrError` with the library's message.

The names of the reference's host functions are mirrored one to one at the
bottom (``forward_3d_ray_driven_siddon`` ... ``tv_norm_gpu``) with the same
argument meaning.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libctrecon.so")

# ctr_status
CTR_OK = 0
STATUS_NAMES = {
    0: "CTR_OK", 1: "CTR_ERR_INVALID_ARGUMENT", 2: "CTR_ERR_BAD_GEOMETRY", 3: "CTR_ERR_OUT_OF_MEMORY",
    4: "CTR_ERR_CUDA", 5: "CTR_ERR_TRAVERSAL_BOUND", 6: "CTR_ERR_TIMEOUT", 7: "CTR_ERR_UNSUPPORTED",
    8: "CTR_ERR_NO_DEVICE", 9: "CTR_ERR_IO",
}
# ctr_dtype (F64: the FP64 reference solver's volumes only)
F32, BF16, F16, F64 = 0, 1, 2, 3
GEOM_ENTRY_F64 = 0x1
BP_ACCUMULATE = 0x1
BP_FOV_MASK = 0x2
GEOM_FAN_SLICES = 0x2
GEOM_PARALLEL = 0x4
GEOM_TBCT = 0x8
GEOM_FAST_SUMS = 0x10
SART_STOCHASTIC_ROUND = 0x1
SART_TILED = 0x2
SART_REFERENCE_BP = 0x4
VOLUME_TILED = 0x8

# every symbol include/ctrecon.h declares
EXPORTED = [
    "ctr_geometry_create", "ctr_geometry_destroy", "ctr_geometry_view_trig", "ctr_forward",
    "ctr_backproject", "ctr_sart_pass", "ctr_sart_views", "ctr_sart_views_noalloc", "ctr_forward_trace", "ctr_fgp_tv", "ctr_fista_momentum",
    "ctr_objective", "ctr_tv_norm", "ctr_l2_norm", "ctr_fdk", "ctr_fdk_projector_frame", "ctr_fdk_backproject",
    "ctr_dot_test", "ctr_solver_create",
    "ctr_solver_destroy", "ctr_solver_set_sinogram", "ctr_solver_set_volume", "ctr_solver_iterate",
    "ctr_solver_get_volume", "ctr_solver_iteration_count", "ctr_solver_save", "ctr_solver_load",
    "ctr_last_error_string", "ctr_convert", "ctr_phantom_voxelize", "ctr_set_default_geometry",
    "Forward_3D_ray_driven_siddon", "Reconstruction_3D_ray_driven_CBCT", "CheckMatchedJointOperator",
    "FGP_denoise_GPUx7_exact", "Reconstruction_FDK", "L2_norm_gpu", "TV_norm_gpu",
    "ctr_io_view_filename", "ctr_io_recon_filename", "ctr_io_objective_filename", "ctr_io_write_raw",
    "ctr_io_read_raw", "ctr_io_read_views", "ctr_io_write_views",
    "ctr_batch_create", "ctr_batch_destroy", "ctr_batch_set_sinogram", "ctr_batch_reset", "ctr_batch_iterate",
    "ctr_batch_get_volume", "ctr_geometry_set_shapes", "ctr_geometry_get_shapes", "ctr_geometry_autotune",
    "ctr_solver_objectives", "ctr_geometry_create_slab", "ctr_geometry_slab", "ctr_forward_partial",
    "ctr_combine_partials", "ctr_sart_update", "ctr_sart_pass_slabs", "ctr_volume_tiling", "ctr_volume_tiled_count",
    "ctr_set_default_devices", "ctr_solver_set_slabs", "ctr_solver_get_volume_f32", "ctr_batch_get_volume_f32",
    "ctr_batch_set_persistent",
]


class CtrError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GeometryDesc(C.Structure):
    """Mirror of ``ctr_geometry_desc``."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("vx", C.c_float), ("vy", C.c_float), ("vz", C.c_float),
        ("nu", C.c_int), ("nv", C.c_int),
        ("du", C.c_float), ("dv", C.c_float),
        ("dso", C.c_float), ("dod", C.c_float), ("offset", C.c_float), ("m_offset", C.c_int),
        ("n_views", C.c_int), ("us_rate", C.c_float), ("initial_angle", C.c_float),
        ("shift_angle", C.c_float), ("flags", C.c_uint), ("n_sources", C.c_int),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("beta", C.c_float), ("lambda_tv", C.c_float), ("fgp_iters", C.c_int), ("fista", C.c_int),
        ("objective", C.c_int), ("use_graph", C.c_int), ("sart_flags", C.c_uint), ("refine", C.c_int),
    ]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the in-tree ``libctrecon.so``; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python gpu_b200/build.py` (the engine has no CPU fallback)")
    lib = C.CDLL(path)
    vp, i, f, d, u = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_uint
    G = C.c_void_p
    sig = {
        "ctr_geometry_create": ([C.POINTER(GeometryDesc), C.POINTER(C.c_void_p)], i),
        "ctr_geometry_destroy": ([G], i),
        "ctr_geometry_view_trig": ([G, i, C.POINTER(f), C.POINTER(f)], i),
        "ctr_forward": ([G, vp, i, vp, i, i, i, vp], i),
        "ctr_backproject": ([G, vp, i, i, vp, i, u, vp], i),
        "ctr_sart_pass": ([G, vp, i, vp, i, f, u, C.c_uint32, vp], i),
        "ctr_sart_views": ([G, vp, i, vp, i, f, u, C.c_uint32, i, i, C.POINTER(f), C.POINTER(f), vp], i),
        "ctr_sart_views_noalloc": ([G, vp, i, vp, i, f, u, C.c_uint32, i, i, vp], i),
        "ctr_forward_trace": ([G, vp, i, vp, vp, vp, vp], i),
        "ctr_fgp_tv": ([G, vp, i, f, i, vp], i),
        "ctr_fista_momentum": ([G, vp, vp, vp, i, f, f, vp], i),
        "ctr_objective": ([G, vp, i, vp, i, C.POINTER(d), C.POINTER(d), vp], i),
        "ctr_tv_norm": ([G, vp, i, C.POINTER(d), vp], i),
        "ctr_l2_norm": ([vp, vp, C.c_int64, C.POINTER(d), vp], i),
        "ctr_fdk": ([G, vp, vp, vp], i),
        "ctr_fdk_backproject": ([G, vp, i, i, vp, vp], i),
        "ctr_fdk_projector_frame": ([G, vp, vp, vp], i),
        "ctr_dot_test": ([G, vp, vp, i, i, C.POINTER(d), C.POINTER(d), vp], i),
        "ctr_solver_create": ([G, i, C.POINTER(SolverParams), C.POINTER(C.c_void_p)], i),
        "ctr_solver_destroy": ([vp], i),
        "ctr_solver_set_sinogram": ([vp, vp, i], i),
        "ctr_solver_set_volume": ([vp, vp, vp], i),
        "ctr_solver_iterate": ([vp, i, vp, vp], i),
        "ctr_solver_get_volume": ([vp, vp, vp], i),
        "ctr_solver_iteration_count": ([vp, C.POINTER(i)], i),
        "ctr_solver_save": ([vp, C.c_char_p, vp], i),
        "ctr_solver_load": ([vp, C.c_char_p, vp], i),
        "ctr_last_error_string": ([], C.c_char_p),
        "ctr_convert": ([vp, i, vp, i, C.c_int64, vp], i),
        "ctr_phantom_voxelize": ([G, vp, i, vp, vp], i),
        "ctr_set_default_geometry": ([C.POINTER(GeometryDesc)], i),
        "Forward_3D_ray_driven_siddon": ([vp, vp], None),
        "Reconstruction_3D_ray_driven_CBCT": ([vp, vp, f], None),
        "CheckMatchedJointOperator": ([vp], None),
        "FGP_denoise_GPUx7_exact": ([vp, f, i], None),
        "Reconstruction_FDK": ([vp, vp], None),
        "L2_norm_gpu": ([vp, vp], d),
        "TV_norm_gpu": ([vp], d),
        "ctr_io_view_filename": ([C.c_char_p, C.c_size_t, i, f, f, i, i], i),
        "ctr_io_recon_filename": ([C.c_char_p, C.c_size_t, C.c_char_p, i, i, i, f, i, f, f, f, f, f, i], i),
        "ctr_io_objective_filename": ([C.c_char_p, C.c_size_t, C.c_char_p, i, f, f, f, f], i),
        "ctr_io_write_raw": ([C.c_char_p, vp, C.c_size_t], i),
        "ctr_io_read_raw": ([C.c_char_p, vp, C.c_size_t, C.c_size_t], i),
        "ctr_io_read_views": ([C.c_char_p, i, i, i, f, f, i, i, vp], i),
        "ctr_io_write_views": ([C.c_char_p, i, i, i, f, f, i, vp], i),
        "ctr_solver_objectives": ([vp, i, i, vp, vp], i),
        "ctr_geometry_set_shapes": ([G, i, i], i),
        "ctr_geometry_get_shapes": ([G, C.POINTER(i), C.POINTER(i)], i),
        "ctr_geometry_autotune": ([G, i, i, C.POINTER(f), C.POINTER(f), vp], i),
        "ctr_batch_create": ([C.POINTER(C.c_void_p), i, i, C.POINTER(SolverParams), C.POINTER(C.c_void_p)], i),
        "ctr_batch_destroy": ([vp], i),
        "ctr_batch_set_sinogram": ([vp, i, vp, i], i),
        "ctr_batch_reset": ([vp, vp], i),
        "ctr_batch_iterate": ([vp, i, vp, vp], i),
        "ctr_batch_get_volume": ([vp, i, vp, vp], i),
        "ctr_geometry_create_slab": ([C.POINTER(GeometryDesc), i, i, C.POINTER(C.c_void_p)], i),
        "ctr_geometry_slab": ([G, C.POINTER(i), C.POINTER(i), C.POINTER(i)], i),
        "ctr_forward_partial": ([G, vp, i, i, vp, u, vp], i),
        "ctr_combine_partials": ([G, vp, i, i, vp, i, vp, vp], i),
        "ctr_sart_update": ([G, vp, i, vp, i, f, u, C.c_uint32, vp], i),
        "ctr_sart_pass_slabs": ([G, i, vp, i, vp, i, f, u, C.c_uint32, i, i, vp], i),
        "ctr_volume_tiling": ([G, vp, vp, i, i, vp], i),
        "ctr_volume_tiled_count": ([G, C.POINTER(C.c_int64)], i),
        "ctr_set_default_devices": ([i], i),
        "ctr_solver_set_slabs": ([vp, i], i),
        "ctr_solver_get_volume_f32": ([vp, vp, vp], i),
        "ctr_batch_get_volume_f32": ([vp, i, vp, vp], i),
        "ctr_batch_set_persistent": ([vp, i], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    return load_library().ctr_last_error_string().decode()


def check(status):
    if status != CTR_OK:
        raise CtrError(status, last_error())


def _ptr(t):
    """Device (torch) or host (numpy) buffer address."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        if not t.is_contiguous():
            raise ValueError("buffer must be contiguous")
        return t.data_ptr()
    if isinstance(t, np.ndarray):
        if not t.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return t.ctypes.data
    return int(t)


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def dtype_code(t) -> int:
    import torch
    dt = t.dtype
    if dt == torch.float32:
        return F32
    if dt == torch.bfloat16:
        return BF16
    if dt == torch.float16:
        return F16
    if dt == torch.float64:
        return F64
    raise TypeError(f"unsupported dtype {dt}")


def make_desc(nx, ny, nz, vx, nu, nv, du, dso, dod, n_views, us_rate=None, initial_angle=0.0,
              shift_angle=0.0, offset=0.0, m_offset=0, entry64=False, vy=0.0, vz=0.0, dv=0.0, ct_style=0,
              n_sources=0, fast_sums=False):
    """ct_style: 0 cone beam, 1 multi-slice fan beam, 2 parallel beam (the
    reference's CT_style); styles 1 and 2 default vz to the detector pitch, as
    the reference does.  ct_style 3: the tetrahedron beam with n_sources
    sources, nv detector rows each (a view has n_sources * nv rows).
    fast_sums: CTR_GEOM_FAST_SUMS (fused ray-sum accumulation)."""
    if us_rate is None:
        us_rate = 360.0 / n_views
    if ct_style in (1, 2) and not vz:
        vz = du
    flags = (GEOM_ENTRY_F64 if entry64 else 0) | {0: 0, 1: GEOM_FAN_SLICES, 2: GEOM_PARALLEL, 3: GEOM_TBCT}[ct_style]
    flags |= GEOM_FAST_SUMS if fast_sums else 0
    return GeometryDesc(nx, ny, nz, vx, vy, vz, nu, nv, du, dv, dso, dod, offset, m_offset, n_views,
                        us_rate, initial_angle, shift_angle, flags, n_sources if ct_style == 3 else 0)


class Geometry:
    """A scan geometry on the current CUDA device (``ctr_geometry``).

    With ``n_slabs`` > 1: slab ``slab`` of the z split of the reference's
    multi-GPU build (``ctr_geometry_create_slab``); its volumes are that slab's
    nz/n_slabs slices; ``slab = -1``: the whole volume as that build's
    row-split projector traverses it."""

    def __init__(self, desc: GeometryDesc, n_slabs: int = 1, slab: int = 0):
        self.lib = load_library()
        self.desc = desc
        self.n_slabs, self.slab = n_slabs, slab
        h = C.c_void_p()
        if n_slabs > 1:
            check(self.lib.ctr_geometry_create_slab(C.byref(desc), n_slabs, slab, C.byref(h)))
        else:
            check(self.lib.ctr_geometry_create(C.byref(desc), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ctr_geometry_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # shapes
    @property
    def vol_shape(self):
        # slab -1: the whole volume (the n-device build's row-split projector)
        nz = self.desc.nz // self.n_slabs if self.slab >= 0 else self.desc.nz
        return (nz, self.desc.ny, self.desc.nx)

    @property
    def first_slice(self):
        """Index in the whole volume of this geometry's first slice."""
        return self.vol_shape[0] * max(self.slab, 0)

    def slab_info(self):
        """(n_slabs, slab, first slice) as the library holds them (``ctr_geometry_slab``)."""
        n, s, k0 = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.ctr_geometry_slab(self.h, C.byref(n), C.byref(s), C.byref(k0)))
        return n.value, s.value, k0.value

    @property
    def view_shape(self):
        """(rows, columns) of one view; the tetrahedron beam's rows are all its sources' bands."""
        d = self.desc
        return (d.nv * (d.n_sources if d.flags & GEOM_TBCT else 1), d.nu)

    @property
    def n_views(self):
        return self.desc.n_views

    def view_trig(self, view):
        s, c = C.c_float(), C.c_float()
        check(self.lib.ctr_geometry_view_trig(self.h, view, C.byref(s), C.byref(c)))
        return s.value, c.value

    # operators (device tensors)
    def forward(self, vol, sino, view_begin=0, view_count=None, stream=None):
        n = self.n_views - view_begin if view_count is None else view_count
        check(self.lib.ctr_forward(self.h, _ptr(vol), dtype_code(vol), _ptr(sino), dtype_code(sino),
                                   view_begin, n, _stream(stream)))
        return sino

    def backproject(self, sino, vol, view_begin=0, view_count=None, flags=0, stream=None):
        n = self.n_views - view_begin if view_count is None else view_count
        check(self.lib.ctr_backproject(self.h, _ptr(sino), view_begin, n, _ptr(vol), dtype_code(vol), flags,
                                       _stream(stream)))
        return vol

    def sart_pass(self, vol, sino, beta, flags=0, seed=0, stream=None):
        check(self.lib.ctr_sart_pass(self.h, _ptr(vol), dtype_code(vol), _ptr(sino), dtype_code(sino), beta, flags,
                                     seed, _stream(stream)))
        return vol

    def sart_views(self, vol, sino, beta, view_begin, view_count, flags=0, seed=0, timed=False, stream=None):
        """SART over a view range; with timed=True returns (fp_ms, bp_ms) summed kernel times."""
        fp, bp = C.c_float(), C.c_float()
        check(self.lib.ctr_sart_views(self.h, _ptr(vol), dtype_code(vol), _ptr(sino), dtype_code(sino), beta, flags,
                                      seed, view_begin, view_count, C.byref(fp) if timed else None,
                                      C.byref(bp) if timed else None, _stream(stream)))
        return (fp.value, bp.value) if timed else None

    # z-slab SART of the multi-GPU build
    def forward_partial(self, vol, view, part, flags=0, stream=None):
        """part (rows, nu, 2) float32 <- this slab's (Sum(len*f), Sum(len)) per ray."""
        check(self.lib.ctr_forward_partial(self.h, _ptr(vol), dtype_code(vol), view, _ptr(part), flags,
                                           _stream(stream)))
        return part

    def combine_partials(self, parts, view, b_view, rays, stream=None):
        """rays (rows, nu, 2) float32 <- (correction, d12) from parts (n, rows, nu, 2) in slab order."""
        check(self.lib.ctr_combine_partials(self.h, _ptr(parts), parts.shape[0], view, _ptr(b_view),
                                            dtype_code(b_view), _ptr(rays), _stream(stream)))
        return rays

    def sart_update(self, vol, rays, view, beta, flags=0, seed=0, stream=None):
        check(self.lib.ctr_sart_update(self.h, _ptr(vol), dtype_code(vol), _ptr(rays), view, beta, flags, seed,
                                       _stream(stream)))
        return vol

    def sart_pass_slabs(self, vol, sino, beta, n_slabs, view_begin=0, view_count=None, flags=0, seed=0,
                        stream=None):
        """The n_slabs-way slab SART on one GPU (vol: the whole volume)."""
        n = self.n_views - view_begin if view_count is None else view_count
        check(self.lib.ctr_sart_pass_slabs(self.h, n_slabs, _ptr(vol), dtype_code(vol), _ptr(sino),
                                           dtype_code(sino), beta, flags, seed, view_begin, n, _stream(stream)))
        return vol

    def tiled_count(self):
        n = C.c_int64()
        check(self.lib.ctr_volume_tiled_count(self.h, C.byref(n)))
        return n.value

    def volume_tiling(self, src, dst, to_tiled=True, stream=None):
        check(self.lib.ctr_volume_tiling(self.h, _ptr(src), _ptr(dst), dtype_code(src), int(to_tiled),
                                         _stream(stream)))
        return dst

    def forward_trace(self, vol, view, nseg, hsh, length, stream=None):
        check(self.lib.ctr_forward_trace(self.h, _ptr(vol), view, _ptr(nseg), _ptr(hsh), _ptr(length),
                                         _stream(stream)))

    def fgp_tv(self, vol, lam, n_iter, stream=None):
        check(self.lib.ctr_fgp_tv(self.h, _ptr(vol), dtype_code(vol), lam, n_iter, _stream(stream)))
        return vol

    def fista_momentum(self, y, x_prev, x, t_prev, t_k, stream=None):
        check(self.lib.ctr_fista_momentum(self.h, _ptr(y), _ptr(x_prev), _ptr(x), dtype_code(y), t_prev, t_k,
                                          _stream(stream)))

    def objective(self, vol, sino, stream=None):
        fid, tv = C.c_double(), C.c_double()
        check(self.lib.ctr_objective(self.h, _ptr(vol), dtype_code(vol), _ptr(sino), dtype_code(sino),
                                     C.byref(fid), C.byref(tv), _stream(stream)))
        return fid.value, tv.value

    def tv_norm(self, vol, stream=None):
        tv = C.c_double()
        check(self.lib.ctr_tv_norm(self.h, _ptr(vol), dtype_code(vol), C.byref(tv), _stream(stream)))
        return tv.value

    def fdk(self, sino, vol, stream=None):
        """vol += FDK in the reference's frame (x and y exchanged against ``forward``)."""
        check(self.lib.ctr_fdk(self.h, _ptr(sino), _ptr(vol), _stream(stream)))
        return vol

    def fdk_projector_frame(self, sino, vol, stream=None):
        """vol += FDK in the projectors' frame (``ctr_fdk_projector_frame``)."""
        check(self.lib.ctr_fdk_projector_frame(self.h, _ptr(sino), _ptr(vol), _stream(stream)))
        return vol

    def fdk_backproject(self, filtered, vol, view_begin=0, view_count=None, stream=None):
        """vol += FDK backprojection of weighted, filtered views (FP32)."""
        n = self.n_views - view_begin if view_count is None else view_count
        check(self.lib.ctr_fdk_backproject(self.h, _ptr(filtered), view_begin, n, _ptr(vol), _stream(stream)))
        return vol

    def dot_test(self, x, y, view_begin=0, view_count=None, stream=None):
        n = self.n_views - view_begin if view_count is None else view_count
        a, b = C.c_double(), C.c_double()
        check(self.lib.ctr_dot_test(self.h, _ptr(x), _ptr(y), view_begin, n, C.byref(a), C.byref(b),
                                    _stream(stream)))
        return a.value, b.value

    def phantom_voxelize(self, params, vol, stream=None):
        p = np.ascontiguousarray(params, np.float64)
        check(self.lib.ctr_phantom_voxelize(self.h, p.ctypes.data, p.shape[0], _ptr(vol), _stream(stream)))
        return vol

    FP_SHAPES = 7
    BP_SHAPES = 6

    def set_shapes(self, fp_shape, bp_shape):
        """Launch shapes of the SART projectors (``ctr_geometry_set_shapes``)."""
        check(self.lib.ctr_geometry_set_shapes(self.h, fp_shape, bp_shape))

    def shapes(self):
        a, b = C.c_int(), C.c_int()
        check(self.lib.ctr_geometry_get_shapes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, vol_dtype=F32, n_views=4, stream=None):
        """Time every projector shape on n_views views and keep the fastest;
        returns {"fp_ms": [...], "bp_ms": {shape: ms}, "fp_shape": s, "bp_shape": s}."""
        fp = (C.c_float * self.FP_SHAPES)()
        bp = (C.c_float * (self.BP_SHAPES + 1))()
        check(self.lib.ctr_geometry_autotune(self.h, vol_dtype, n_views, fp, bp, _stream(stream)))
        f, b = self.shapes()
        return {"fp_ms": list(fp), "bp_ms": {s - 1: bp[s] for s in range(self.BP_SHAPES + 1)}, "fp_shape": f,
                "bp_shape": b}


def l2_norm(a, b, stream=None):
    out = C.c_double()
    check(load_library().ctr_l2_norm(_ptr(a), _ptr(b), a.numel(), C.byref(out), _stream(stream)))
    return out.value


def convert(src, dst, stream=None):
    check(load_library().ctr_convert(_ptr(src), dtype_code(src), _ptr(dst), dtype_code(dst), src.numel(),
                                     _stream(stream)))
    return dst


class Solver:
    """SART + FISTA + FGP-TV outer loop on device buffers (``ctr_solver``).

    ``beta`` is the SART relaxation.  The reference's FISTA loop uses its step
    2/Lip_con = 2/32 = 0.0625 (V63/main_recon.cu:58,161), and its FGP lambda is
    beta * lambda_tv.  The default 0.8 suits plain SART (``fista=False``); under
    FISTA it makes the iteration diverge after a few passes on a 256^3 /
    360-view scan, so pass the reference's step there.

    ``refine=True`` (or 1, with a BF16/F16 ``vol_dtype``): mixed-precision
    iterative refinement -- FP32 FISTA state, 16-bit copies for the
    projectors, each SART pass accumulated into a 16-bit correction against
    the FP32 residual.  ``refine=2``: the same with the correction in FP32.
    ``vol_dtype=F64``: the FP64 reference solver (FP64 volumes)."""

    def __init__(self, geom: Geometry, vol_dtype=F32, beta=0.8, lambda_tv=0.0, fgp_iters=20, fista=True,
                 objective=True, use_graph=True, sart_flags=0, refine=False):
        self.geom = geom
        self.lib = geom.lib
        self.vol_dtype = vol_dtype
        self.params = SolverParams(beta, lambda_tv, fgp_iters, int(fista), int(objective), int(use_graph),
                                   sart_flags, int(refine))
        h = C.c_void_p()
        check(self.lib.ctr_solver_create(geom.h, vol_dtype, C.byref(self.params), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ctr_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sinogram(self, sino):
        self._sino = sino  # keep the borrowed buffer alive
        check(self.lib.ctr_solver_set_sinogram(self.h, _ptr(sino), dtype_code(sino)))

    def set_volume(self, vol=None, stream=None):
        check(self.lib.ctr_solver_set_volume(self.h, _ptr(vol), _stream(stream)))

    def iterate(self, n, stream=None, objectives=True):
        """n iterations; returns their [TV, fidelity, objective] rows, or None
        with objectives=False (the last objective is then projected inside the
        next call's first SART pass, or by ``objectives()``)."""
        if not objectives:
            check(self.lib.ctr_solver_iterate(self.h, n, None, _stream(stream)))
            return None
        obj = np.zeros(3 * max(n, 1), np.float64)
        check(self.lib.ctr_solver_iterate(self.h, n, obj.ctypes.data, _stream(stream)))
        return obj[: 3 * n].reshape(n, 3)

    def set_slabs(self, n_slabs):
        """The SART pass of the reference's n_slabs-device build (``ctr_solver_set_slabs``)."""
        check(self.lib.ctr_solver_set_slabs(self.h, n_slabs))

    def objectives(self, first, count, stream=None):
        """Objective history rows of iterations first..first+count-1 (1-based)."""
        obj = np.zeros(3 * max(count, 1), np.float64)
        check(self.lib.ctr_solver_objectives(self.h, first, count, obj.ctypes.data, _stream(stream)))
        return obj[: 3 * count].reshape(count, 3)

    def get_volume(self, out, stream=None):
        check(self.lib.ctr_solver_get_volume(self.h, _ptr(out), _stream(stream)))
        return out

    def get_volume_f32(self, out, stream=None):
        """The estimate as FP32: a refinement solver's FP32 x_k, otherwise the stored one converted."""
        check(self.lib.ctr_solver_get_volume_f32(self.h, _ptr(out), _stream(stream)))
        return out

    @property
    def iteration(self):
        k = C.c_int()
        check(self.lib.ctr_solver_iteration_count(self.h, C.byref(k)))
        return k.value

    def save(self, path, stream=None):
        check(self.lib.ctr_solver_save(self.h, str(path).encode(), _stream(stream)))

    def load(self, path, stream=None):
        check(self.lib.ctr_solver_load(self.h, str(path).encode(), _stream(stream)))


class Batch:
    """Many scans iterated together, one CUDA graph launch per iteration (``ctr_batch``)."""

    def __init__(self, geoms, vol_dtype=F32, beta=0.8, lambda_tv=0.0, fgp_iters=20, fista=True, objective=True,
                 sart_flags=0, refine=False):
        self.geoms = list(geoms)
        self.lib = load_library()
        self.params = SolverParams(beta, lambda_tv, fgp_iters, int(fista), int(objective), 1, sart_flags,
                                   int(refine))
        arr = (C.c_void_p * len(self.geoms))(*[g.h.value for g in self.geoms])
        h = C.c_void_p()
        check(self.lib.ctr_batch_create(arr, len(self.geoms), vol_dtype, C.byref(self.params), C.byref(h)))
        self.h = h
        self._sinos = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.ctr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sinogram(self, scan, sino):
        self._sinos[scan] = sino
        check(self.lib.ctr_batch_set_sinogram(self.h, scan, _ptr(sino), dtype_code(sino)))

    def reset(self, stream=None):
        check(self.lib.ctr_batch_reset(self.h, _stream(stream)))

    def iterate(self, n, stream=None):
        obj = np.zeros(len(self.geoms) * max(n, 1) * 3, np.float64)
        check(self.lib.ctr_batch_iterate(self.h, n, obj.ctypes.data, _stream(stream)))
        return obj[: len(self.geoms) * n * 3].reshape(len(self.geoms), n, 3)

    def get_volume(self, scan, out, stream=None):
        check(self.lib.ctr_batch_get_volume(self.h, scan, _ptr(out), _stream(stream)))
        return out

    def get_volume_f32(self, scan, out, stream=None):
        check(self.lib.ctr_batch_get_volume_f32(self.h, scan, _ptr(out), _stream(stream)))
        return out

    def set_persistent(self, on=True):
        """Every scan's SART views in one persistent launch per iteration (``ctr_batch_set_persistent``)."""
        check(self.lib.ctr_batch_set_persistent(self.h, int(on)))


# ---------------------------------------------------------------------------
# The reference driver's file formats
# ---------------------------------------------------------------------------

def view_filename(view, us_rate, initial_angle=0.0, tomo=0, n_views=0):
    buf = C.create_string_buffer(64)
    check(load_library().ctr_io_view_filename(buf, 64, view, us_rate, initial_angle, tomo, n_views))
    return buf.value.decode()


def recon_filename(object_name, nx, ny, nz, voxel_um, n_views, initial_angle, end_angle, lambda_tv, lambda_l1,
                   lip, iteration=-1):
    buf = C.create_string_buffer(512)
    check(load_library().ctr_io_recon_filename(buf, 512, object_name.encode(), nx, ny, nz, voxel_um, n_views,
                                               initial_angle, end_angle, lambda_tv, lambda_l1, lip, iteration))
    return buf.value.decode()


def objective_filename(object_name, n_views, initial_angle, end_angle, lambda_tv, lip):
    buf = C.create_string_buffer(512)
    check(load_library().ctr_io_objective_filename(buf, 512, object_name.encode(), n_views, initial_angle,
                                                   end_angle, lambda_tv, lip))
    return buf.value.decode()


def write_raw(path, arr):
    a = np.ascontiguousarray(arr)
    check(load_library().ctr_io_write_raw(str(path).encode(), a.ctypes.data, a.nbytes))


def read_raw(path, shape, dtype=np.float32, offset=0):
    a = np.empty(shape, dtype)
    check(load_library().ctr_io_read_raw(str(path).encode(), a.ctypes.data, a.nbytes, offset))
    return a


def write_views(directory, proj, us_rate, initial_angle=0.0, tomo=0):
    p = np.ascontiguousarray(proj, np.float32)
    check(load_library().ctr_io_write_views(str(directory).encode(), p.shape[2], p.shape[1], p.shape[0], us_rate,
                                            initial_angle, tomo, p.ctypes.data))


def read_views(directory, nu, nv, n_views, us_rate, initial_angle=0.0, tomo=0, row_offset=0):
    p = np.empty((n_views, nv, nu), np.float32)
    check(load_library().ctr_io_read_views(str(directory).encode(), nu, nv, n_views, us_rate, initial_angle, tomo,
                                           row_offset, p.ctypes.data))
    return p


# ---------------------------------------------------------------------------
# The reference's host entry points (V63/host_*.c[u|pp]), same names and
# argument meaning; host numpy arrays are updated in place like the reference.
# ---------------------------------------------------------------------------

def set_default_devices(n: int):
    """Number_of_Devices of the reference build the host functions stand in for."""
    check(load_library().ctr_set_default_devices(n))


def set_default_geometry(desc: GeometryDesc):
    check(load_library().ctr_set_default_geometry(C.byref(desc)))


def _after_void():
    msg = last_error()
    if msg:
        raise CtrError(-1, msg)


def forward_3d_ray_driven_siddon(h_volume: np.ndarray, h_proj_data: np.ndarray):
    load_library().Forward_3D_ray_driven_siddon(_ptr(h_volume), _ptr(h_proj_data))
    _after_void()


def reconstruction_3d_ray_driven_cbct(h_volume: np.ndarray, h_proj_data: np.ndarray, beta: float):
    load_library().Reconstruction_3D_ray_driven_CBCT(_ptr(h_volume), _ptr(h_proj_data), beta)
    _after_void()


def check_matched_joint_operator(h_volume: np.ndarray):
    load_library().CheckMatchedJointOperator(_ptr(h_volume))
    _after_void()


def fgp_denoise_gpux7_exact(h_f: np.ndarray, lam: float, n_iter: int):
    load_library().FGP_denoise_GPUx7_exact(_ptr(h_f), lam, n_iter)
    _after_void()


def reconstruction_fdk(h_volume: np.ndarray, h_proj_data: np.ndarray):
    load_library().Reconstruction_FDK(_ptr(h_volume), _ptr(h_proj_data))
    _after_void()


def l2_norm_gpu(a, b) -> float:
    r = load_library().L2_norm_gpu(_ptr(a), _ptr(b))
    _after_void()
    return r


def tv_norm_gpu(vol) -> float:
    r = load_library().TV_norm_gpu(_ptr(vol))
    _after_void()
    return r
