"""ctypes wrappers over the CPU oracle libraries (test infrastructure only).

``Oracle`` wraps the C restatement (``libctoracle.so``); ``RefOracle`` wraps the
reference's own kernels compiled for the CPU (``_ref/libctref.so``).  Both take
and return numpy arrays in the reference's layouts: volume ``[Z][N][M]``, one
view ``[Z_prj][R]``, sinogram ``[views][Z_prj][R]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libctoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libctref.so")
# the reference fixes CT_style at compile time: one build per style
# (3: the tetrahedron-beam program's kernels)
REF_SO_STYLE = {0: REF_SO, 1: os.path.join(HERE, "_ref", "libctref_fbct.so"),
                2: os.path.join(HERE, "_ref", "libctref_pbct.so"), 3: os.path.join(HERE, "_ref", "libctref_tbct.so")}
# the tetrahedron-beam program's multi-GPU build (its own kernels)
REF_SO_TBCT_MULTI = os.path.join(HERE, "_ref", "libctref_tbct_multi.so")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


class OgDesc(C.Structure):
    """Mirror of ``og_desc`` in ct_oracle.h."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("nu", C.c_int), ("nv", C.c_int), ("nviews", C.c_int),
        ("vx", C.c_float), ("vy", C.c_float), ("vz", C.c_float),
        ("du", C.c_float), ("dv", C.c_float),
        ("dso", C.c_float), ("dod", C.c_float),
        ("offset", C.c_float), ("m_offset", C.c_int),
        ("us_rate", C.c_float), ("initial_angle", C.c_float), ("shift_angle", C.c_float),
        ("ct_style", C.c_int), ("n_sources", C.c_int),
        ("n_slabs", C.c_int), ("slab", C.c_int),
    ]


class OgGeom(C.Structure):
    _fields_ = [
        ("d", OgDesc),
        ("inv_vx", C.c_float), ("inv_vy", C.c_float), ("inv_vz", C.c_float),
        ("bx", C.c_float), ("by", C.c_float), ("bz", C.c_float),
        ("ymin", C.c_float), ("zmin", C.c_float),
        ("srcx", C.c_float), ("srcy", C.c_float), ("srcz", C.c_float),
        ("zmax", C.c_float), ("zsrc0", C.c_float), ("zsrc_dz", C.c_float), ("rows", C.c_int),
        ("k0", C.c_int), ("bz_ref", C.c_float), ("zpar_kr", C.c_int), ("row_lo", C.c_int), ("row_hi", C.c_int),
        ("loop_eps", C.c_float),
    ]


def make_desc(nx, ny, nz, nu, nv, nviews, vx, du, dso, dod, us_rate=None,
              initial_angle=0.0, shift_angle=0.0, offset=0.0, m_offset=0, ct_style=0, vz=None,
              n_sources=0):
    """ct_style 1 and 2 take the reference's z pitch, volumn_z = Detector_pixel_x
    (V63/main_recon.cu:96), unless vz is given.  ct_style 3 is the tetrahedron
    beam with n_sources sources, nv detector rows each (volumn_z = volumn_x)."""
    if us_rate is None:
        us_rate = 360.0 / nviews
    if vz is None:
        vz = du if ct_style in (1, 2) else vx
    return OgDesc(nx, ny, nz, nu, nv, nviews, vx, vx, vz, du, du, dso, dod,
                  offset, m_offset, us_rate, initial_angle, shift_angle, ct_style,
                  n_sources if ct_style == 3 else 0)


def slab_desc(desc: OgDesc, n_slabs: int, slab: int) -> OgDesc:
    """The description of slab ``slab`` of the ``n_slabs``-way z split of the
    multi-GPU build (its kernels take the whole scan's constants plus the
    device index); ``slab = -1``: the whole volume as that build's row-split
    projector traverses it."""
    d = OgDesc()
    C.pointer(d)[0] = desc
    d.n_slabs, d.slab = n_slabs, slab
    return d


def build():
    """Compile the oracle libraries (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    if not os.path.exists(path):
        build()
    return C.CDLL(path)


class Oracle:
    """The C restatement of the reference path."""

    def __init__(self, desc: OgDesc):
        self.lib = lib = _load(ORACLE_SO)
        self.desc = desc
        self.g = OgGeom()
        lib.og_init.argtypes = [C.POINTER(OgGeom), C.POINTER(OgDesc)]
        if lib.og_init(C.byref(self.g), C.byref(desc)) != 0:
            raise ValueError("bad geometry")
        G = C.POINTER(OgGeom)
        f, i, d = C.c_float, C.c_int, C.c_double
        sig = {
            "og_view_trig": [G, i, i, C.POINTER(f), C.POINTER(f)],
            "og_forward_view": [G, _f32p, f, f, i, C.c_void_p, _f32p, i],
            "og_forward_trace": [G, _f32p, f, f, i, _i32p, _u64p, _f32p],
            "og_forward_view_f64": [G, _f64p, d, d, _f64p],
            "og_backproject_ref": [G, _f32p, _f32p, f, f, f, i],
            "og_adjoint_view": [G, _f32p, f, f, i, _f64p, C.c_void_p],
            "og_adjoint_view_f64": [G, _f64p, d, d, _f64p],
            "og_fov_masked": [G, i, i],
            "og_sart_pass_ref": [G, _f32p, _f32p, f],
            "og_sart_pass_matched": [G, _f32p, _f32p, f],
            "og_sart_pass_f64": [G, _f64p, _f64p, d],
            "og_backproject_gather": [G, _f32p, _f32p, f, f, f],
            "og_sart_pass_gather": [G, _f32p, _f32p, f],
            "og_fgp": [i, i, i, _f32p, f, i, _f32p],
            "og_fgp_f64": [i, i, i, _f64p, d, i, _f64p],
            "og_tv_norm": [i, i, i, _f32p],
            "og_l2_norm": [_f32p, _f32p, C.c_longlong],
            "og_fista_momentum": [C.c_longlong, _f32p, _f32p, _f32p, f, f],
            "og_fdk_weight": [G, _f32p, _f32p, i],
            "og_ramp_kernel": [G, _f64p],
            "og_ramp_filter": [G, _f32p, _f32p, i],
            "og_ramp_filter_dft": [G, _f32p, _f32p, i],
            "og_fdk_bp_view": [G, _f32p, _f32p, f, f],
            "og_fdk": [G, _f32p, _f32p],
            "og_phantom_voxelize": [G, _f64p, i, _f32p],
            "og_phantom_project": [G, _f64p, i, d, d, _f32p],
            "og_forward_partial": [G, _f32p, f, f, _f32p, _f32p],
            "og_combine_partials": [G, i, _f32p, _f32p, _f32p, _f32p],
            "og_sart_pass_slabs": [C.POINTER(OgDesc), _f32p, _f32p, f, i, i, i],
        }
        for name, args in sig.items():
            getattr(lib, name).argtypes = args
        for name in ("og_tv_norm", "og_l2_norm"):
            getattr(lib, name).restype = C.c_double
        self.gp = C.byref(self.g)

    # shapes
    @property
    def vol_shape(self):
        d = self.desc
        return (d.nz, d.ny, d.nx)

    @property
    def view_shape(self):
        """(rows, columns) of one view: N_source bands of Z_prj rows for ct_style 3."""
        return (self.g.rows, self.desc.nu)

    def trig(self, view, fdk=False):
        s, c = C.c_float(), C.c_float()
        self.lib.og_view_trig(self.gp, view, int(fdk), C.byref(s), C.byref(c))
        return s.value, c.value

    def forward_view(self, vol, view, command=0, b=None, entry64=False):
        s, c = self.trig(view)
        out = np.zeros(self.view_shape, np.float32)
        bp = None if b is None else np.ascontiguousarray(b, np.float32).ctypes.data
        bb = None if b is None else np.ascontiguousarray(b, np.float32)
        self.lib.og_forward_view(self.gp, np.ascontiguousarray(vol, np.float32), s, c, command,
                                 bb.ctypes.data if bb is not None else None, out, int(entry64))
        del bp
        return out

    def forward(self, vol, views=None, entry64=False):
        views = range(self.desc.nviews) if views is None else views
        return np.stack([self.forward_view(vol, j, 0, entry64=entry64) for j in views])

    def forward_trace(self, vol, view, entry64=False):
        s, c = self.trig(view)
        n = np.zeros(self.view_shape, np.int32)
        h = np.zeros(self.view_shape, np.uint64)
        ln = np.zeros(self.view_shape, np.float32)
        self.lib.og_forward_trace(self.gp, np.ascontiguousarray(vol, np.float32), s, c,
                                  int(entry64), n, h, ln)
        return n, h, ln

    def forward_view_f64(self, vol, view):
        t = -((view * self.desc.us_rate + self.desc.initial_angle) + self.desc.shift_angle) * np.pi / 180.0
        out = np.zeros(self.view_shape, np.float64)
        self.lib.og_forward_view_f64(self.gp, np.ascontiguousarray(vol, np.float64),
                                     np.sin(t), np.cos(t), out)
        return out

    def backproject_ref(self, vol, corr, view, beta=1.0, command=1):
        s, c = self.trig(view)
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_backproject_ref(self.gp, vol, np.ascontiguousarray(corr, np.float32),
                                    beta, s, c, command)
        return vol

    def adjoint_view(self, y, view, thresh=False, want_len=False):
        s, c = self.trig(view)
        acc = np.zeros(self.vol_shape, np.float64)
        lacc = np.zeros(self.vol_shape, np.float64) if want_len else None
        self.lib.og_adjoint_view(self.gp, np.ascontiguousarray(y, np.float32), s, c, int(thresh),
                                 acc, lacc.ctypes.data if lacc is not None else None)
        return (acc, lacc) if want_len else acc

    def adjoint(self, sino, views=None):
        views = range(self.desc.nviews) if views is None else views
        acc = np.zeros(self.vol_shape, np.float64)
        for k, j in enumerate(views):
            acc += self.adjoint_view(sino[k], j)
        return acc

    def adjoint_view_f64(self, y, view):
        t = -((view * self.desc.us_rate + self.desc.initial_angle) + self.desc.shift_angle) * np.pi / 180.0
        acc = np.zeros(self.vol_shape, np.float64)
        self.lib.og_adjoint_view_f64(self.gp, np.ascontiguousarray(y, np.float64), np.sin(t), np.cos(t), acc)
        return acc

    def fov_mask(self):
        d = self.desc
        m = np.zeros((d.ny, d.nx), bool)
        for j in range(d.ny):
            for i in range(d.nx):
                m[j, i] = bool(self.lib.og_fov_masked(self.gp, i, j))
        return m

    def sart_pass_ref(self, vol, sino, beta):
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_sart_pass_ref(self.gp, vol, np.ascontiguousarray(sino, np.float32), beta)
        return vol

    def sart_pass_matched(self, vol, sino, beta):
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_sart_pass_matched(self.gp, vol, np.ascontiguousarray(sino, np.float32), beta)
        return vol

    def backproject_gather(self, vol, corr, view, beta):
        s, c = self.trig(view)
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_backproject_gather(self.gp, vol, np.ascontiguousarray(corr, np.float32), beta, s, c)
        return vol

    def sart_pass_gather(self, vol, sino, beta):
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_sart_pass_gather(self.gp, vol, np.ascontiguousarray(sino, np.float32), beta)
        return vol

    def sart_pass_f64(self, vol, sino, beta):
        vol = np.ascontiguousarray(vol, np.float64).copy()
        self.lib.og_sart_pass_f64(self.gp, vol, np.ascontiguousarray(sino, np.float64), beta)
        return vol

    def forward_partial(self, vol, view):
        """On a slab description: the slab's (Sum(len*f), Sum(len)) per ray."""
        s, c = self.trig(view)
        w = np.zeros(self.view_shape, np.float32)
        ln = np.zeros(self.view_shape, np.float32)
        self.lib.og_forward_partial(self.gp, np.ascontiguousarray(vol, np.float32), s, c, w, ln)
        return w, ln

    def combine_partials(self, wsum, lsum, b):
        """The SART correction of the parts [n_parts][rows][R], added in order."""
        wsum = np.ascontiguousarray(wsum, np.float32)
        out = np.zeros(self.view_shape, np.float32)
        self.lib.og_combine_partials(self.gp, wsum.shape[0], wsum, np.ascontiguousarray(lsum, np.float32),
                                     np.ascontiguousarray(b, np.float32), out)
        return out

    def sart_pass_slabs(self, vol, sino, beta, n_slabs, v0=0, nv=None, engine=False):
        """Views [v0, v0+nv) of the n_slabs-way slab SART on the whole volume."""
        nv = self.desc.nviews - v0 if nv is None else nv
        vol = np.ascontiguousarray(vol, np.float32).copy()
        d = slab_desc(self.desc, n_slabs, 0)
        if self.lib.og_sart_pass_slabs(C.byref(d), vol, np.ascontiguousarray(sino, np.float32), beta, v0, nv,
                                       int(engine)) != 0:
            raise ValueError("the scan does not split into %d slabs" % n_slabs)
        return vol

    def fgp(self, f, lam, iters):
        d = self.desc
        out = np.zeros(self.vol_shape, np.float32)
        self.lib.og_fgp(d.nx, d.ny, d.nz, np.ascontiguousarray(f, np.float32), lam, iters, out)
        return out

    def fgp_f64(self, f, lam, iters):
        d = self.desc
        out = np.zeros(self.vol_shape, np.float64)
        self.lib.og_fgp_f64(d.nx, d.ny, d.nz, np.ascontiguousarray(f, np.float64), lam, iters, out)
        return out

    def tv_norm(self, vol):
        d = self.desc
        return self.lib.og_tv_norm(d.nx, d.ny, d.nz, np.ascontiguousarray(vol, np.float32))

    def l2_norm(self, a, b):
        a = np.ascontiguousarray(a, np.float32)
        return self.lib.og_l2_norm(a, np.ascontiguousarray(b, np.float32), a.size)

    def fista_momentum(self, y, xprev, x, t_prev, t_k):
        y = np.ascontiguousarray(y, np.float32).copy()
        xprev = np.ascontiguousarray(xprev, np.float32).copy()
        self.lib.og_fista_momentum(y.size, y, xprev, np.ascontiguousarray(x, np.float32), t_prev, t_k)
        return y, xprev

    def fdk_weight(self, sino):
        sino = np.ascontiguousarray(sino, np.float32)
        out = np.zeros_like(sino)
        self.lib.og_fdk_weight(self.gp, sino, out, sino.shape[0])
        return out

    def ramp_kernel(self):
        h = np.zeros(2 * self.desc.nu - 1, np.float64)
        self.lib.og_ramp_kernel(self.gp, h)
        return h

    def ramp_filter(self, rows, dft=False):
        rows = np.ascontiguousarray(rows, np.float32)
        out = np.zeros_like(rows)
        nrows = rows.size // self.desc.nu
        (self.lib.og_ramp_filter_dft if dft else self.lib.og_ramp_filter)(self.gp, rows, out, nrows)
        return out

    def fdk_bp_view(self, vol, proj, view):
        s, c = self.trig(view, fdk=True)
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.og_fdk_bp_view(self.gp, vol, np.ascontiguousarray(proj, np.float32), s, c)
        return vol

    def fdk(self, sino):
        vol = np.zeros(self.vol_shape, np.float32)
        self.lib.og_fdk(self.gp, np.ascontiguousarray(sino, np.float32), vol)
        return vol

    def phantom(self, params):
        vol = np.zeros(self.vol_shape, np.float32)
        p = np.ascontiguousarray(params, np.float64)
        self.lib.og_phantom_voxelize(self.gp, p, p.shape[0], vol)
        return vol

    def phantom_sinogram(self, params, views=None):
        views = range(self.desc.nviews) if views is None else views
        p = np.ascontiguousarray(params, np.float64)
        out = []
        for j in views:
            t = -((j * self.desc.us_rate + self.desc.initial_angle) + self.desc.shift_angle) * np.pi / 180.0
            o = np.zeros(self.view_shape, np.float32)
            self.lib.og_phantom_project(self.gp, p, p.shape[0], np.sin(t), np.cos(t), o)
            out.append(o)
        return np.stack(out)


class RefOracle:
    """The reference's own kernels compiled for the CPU (``_ref/libctref.so``)."""

    def __init__(self, desc: OgDesc, multi: bool = False):
        """multi: the tetrahedron-beam program's multi-GPU build (its slab calls)."""
        so = REF_SO_TBCT_MULTI if multi and desc.ct_style == 3 else REF_SO_STYLE[desc.ct_style]
        if not os.path.exists(so):
            raise FileNotFoundError(so)
        self.lib = lib = C.CDLL(so)
        self.desc = desc
        f, i = C.c_float, C.c_int
        sig = {
            "ref_set_geometry": [C.POINTER(OgDesc)],
            "ref_view_trig": [i, i, C.POINTER(f), C.POINTER(f)],
            "ref_forward_view": [_f32p, _f32p, C.c_void_p, f, f, i],
            "ref_backproject_view": [_f32p, _f32p, f, f, f, i],
            "ref_sart_views": [_f32p, _f32p, f, i, i],
            "ref_fgp": [_f32p, f, i],
            "ref_tv_norm": [_f32p],
            "ref_l2_norm": [_f32p, _f32p, i],
            "ref_fdk_weight": [_f32p, _f32p, i],
            "ref_ramp_filter": [_f32p, _f32p, i],
            "ref_fdk_bp_view": [_f32p, _f32p, f, f],
            "ref_slab_forward_view": [i, i, _f32p, _f32p, _f32p, f, f],
            "ref_combine_view": [i, _f32p, _f32p, _f32p, _f32p],
            "ref_slab_backproject_view": [i, i, _f32p, _f32p, f, f, f, i],
            "ref_sart_views_slabs": [i, _f32p, _f32p, f, i, i],
            "ref_forward_view_split": [i, _f32p, _f32p, f, f],
        }
        for name, args in sig.items():
            if hasattr(lib, name):   # the tetrahedron-beam build has the projectors only
                getattr(lib, name).argtypes = args
        for name in ("ref_tv_norm", "ref_l2_norm"):
            if hasattr(lib, name):
                getattr(lib, name).restype = C.c_double
        self._set()

    def _set(self):
        if self.lib.ref_set_geometry(C.byref(self.desc)) != 0:
            raise ValueError("geometry not representable by the reference")

    @property
    def vol_shape(self):
        d = self.desc
        return (d.nz, d.ny, d.nx)

    @property
    def view_shape(self):
        d = self.desc
        return (d.nv * (d.n_sources if d.ct_style == 3 else 1), d.nu)

    def trig(self, view, fdk=False):
        s, c = C.c_float(), C.c_float()
        self.lib.ref_view_trig(view, int(fdk), C.byref(s), C.byref(c))
        return s.value, c.value

    def forward_view(self, vol, view, command=0, b=None):
        self._set()
        s, c = self.trig(view)
        out = np.zeros(self.view_shape, np.float32)
        bb = None if b is None else np.ascontiguousarray(b, np.float32)
        self.lib.ref_forward_view(np.ascontiguousarray(vol, np.float32), out,
                                  bb.ctypes.data if bb is not None else None, s, c, command)
        return out

    def backproject_view(self, vol, corr, view, beta=1.0, command=1):
        self._set()
        s, c = self.trig(view)
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.ref_backproject_view(vol, np.ascontiguousarray(corr, np.float32), beta, s, c, command)
        return vol

    def sart(self, vol, sino, beta, v0=0, nv=None):
        self._set()
        nv = self.desc.nviews - v0 if nv is None else nv
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.ref_sart_views(vol, np.ascontiguousarray(sino, np.float32), beta, v0, nv)
        return vol

    # the multi-GPU build with Number_of_Devices = D (volume: the D slabs back to back)
    def _slab_vol(self, D):
        d = self.desc
        return (d.nz // D, d.ny, d.nx)

    def slab_forward_view(self, vol_slab, D, sub, view):
        """forward_ray_driven_3d_kernel_correction_separate: (weightedLen, sumLen)."""
        self._set()
        s, c = self.trig(view)
        w = np.zeros(self.view_shape, np.float32)
        ln = np.zeros(self.view_shape, np.float32)
        if self.lib.ref_slab_forward_view(D, sub, np.ascontiguousarray(vol_slab, np.float32), ln, w, s, c) != 0:
            raise ValueError("no %d-way split" % D)
        return w, ln

    def combine_view(self, wsum, lsum, b):
        self._set()
        wsum = np.ascontiguousarray(wsum, np.float32)
        out = np.zeros(self.view_shape, np.float32)
        if self.lib.ref_combine_view(wsum.shape[0], np.ascontiguousarray(lsum, np.float32), wsum,
                                     np.ascontiguousarray(b, np.float32), out) != 0:
            raise ValueError("no split")
        return out

    def slab_backproject_view(self, vol_slab, corr, D, sub, view, beta=1.0, command=1):
        self._set()
        s, c = self.trig(view)
        vol = np.ascontiguousarray(vol_slab, np.float32).copy()
        if self.lib.ref_slab_backproject_view(D, sub, vol, np.ascontiguousarray(corr, np.float32), beta, s, c,
                                              command) != 0:
            raise ValueError("no %d-way split" % D)
        return vol

    def sart_slabs(self, vol, sino, beta, D, v0=0, nv=None):
        self._set()
        nv = self.desc.nviews - v0 if nv is None else nv
        vol = np.ascontiguousarray(vol, np.float32).copy()
        if self.lib.ref_sart_views_slabs(D, vol, np.ascontiguousarray(sino, np.float32), beta, v0, nv) != 0:
            raise ValueError("no %d-way split" % D)
        return vol

    def forward_view_split(self, vol, D, view):
        self._set()
        s, c = self.trig(view)
        out = np.zeros(self.view_shape, np.float32)
        if self.lib.ref_forward_view_split(D, np.ascontiguousarray(vol, np.float32), out, s, c) != 0:
            raise ValueError("no %d-way split" % D)
        return out

    def fgp(self, f, lam, iters):
        self._set()
        f = np.ascontiguousarray(f, np.float32).copy()
        self.lib.ref_fgp(f, lam, iters)
        return f

    def tv_norm(self, vol):
        self._set()
        return self.lib.ref_tv_norm(np.ascontiguousarray(vol, np.float32))

    def l2_norm(self, a, b):
        self._set()
        a = np.ascontiguousarray(a, np.float32).copy()
        return self.lib.ref_l2_norm(a, np.ascontiguousarray(b, np.float32), a.size // (self.desc.nu * self.desc.nv))

    def fdk_weight(self, sino):
        self._set()
        sino = np.ascontiguousarray(sino, np.float32)
        out = np.zeros_like(sino)
        self.lib.ref_fdk_weight(sino, out, sino.shape[0])
        return out

    def ramp_filter(self, rows):
        self._set()
        rows = np.ascontiguousarray(rows, np.float32)
        out = np.zeros_like(rows)
        self.lib.ref_ramp_filter(rows, out, rows.size // self.desc.nu)
        return out

    def fdk_bp_view(self, vol, proj, view):
        self._set()
        s, c = self.trig(view, fdk=True)
        vol = np.ascontiguousarray(vol, np.float32).copy()
        self.lib.ref_fdk_bp_view(vol, np.ascontiguousarray(proj, np.float32), s, c)
        return vol


def random_ellipsoids(rng, n, center_range, axes_range, mu_range):
    """Seeded ellipsoid parameters: n x 10 (cx,cy,cz, ax,ay,az, phi,theta,psi, mu)."""
    p = np.zeros((n, 10))
    p[:, 0:3] = rng.uniform(-center_range, center_range, (n, 3))
    p[:, 3:6] = rng.uniform(axes_range[0], axes_range[1], (n, 3))
    p[:, 6:9] = rng.uniform(0, 2 * np.pi, (n, 3))
    p[:, 9] = rng.uniform(mu_range[0], mu_range[1], n)
    return p
