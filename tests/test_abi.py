"""The C-ABI library loads, exports every entry point include/ctrecon.h
declares, and rejects bad arguments before touching a device."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "ctrecon.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


def test_header_and_binding_agree():
    import gpu_b200
    assert sorted(gpu_b200.EXPORTED) == declared_functions()


def test_library_exports_every_symbol():
    import gpu_b200
    lib = gpu_b200.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    # the shared object is the in-tree build
    assert os.path.dirname(gpu_b200.LIB_PATH) == os.path.join(ROOT, "gpu_b200")


def test_argument_errors_without_device():
    import gpu_b200
    from gpu_b200 import ctrecon
    lib = gpu_b200.load_library()
    assert lib.ctr_forward(None, None, 0, None, 0, 0, 1, None) == 1
    assert "NULL" in gpu_b200.last_error()
    assert lib.ctr_geometry_create(None, None) == 1
    d = ctrecon.make_desc(0, 8, 8, 1.0, 8, 8, 1.0, 1000.0, -500.0, 4)
    h = C.c_void_p()
    assert lib.ctr_geometry_create(C.byref(d), C.byref(h)) == 2       # CTR_ERR_BAD_GEOMETRY
    d = ctrecon.make_desc(8, 8, 8, 1.0, 8, 8, 1.0, 1000.0, 2000.0, 4)  # detector behind the source
    assert lib.ctr_geometry_create(C.byref(d), C.byref(h)) == 2
    d = ctrecon.make_desc(8, 8, 8, float("nan"), 8, 8, 1.0, 1000.0, -500.0, 4)
    assert lib.ctr_geometry_create(C.byref(d), C.byref(h)) == 2
    assert lib.ctr_convert(None, 0, None, 0, 4, None) == 1
    assert lib.ctr_l2_norm(None, None, 4, None, None) == 1


def test_no_device_reported_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import gpu_b200
    from gpu_b200 import ctrecon
    d = ctrecon.make_desc(8, 8, 8, 1.0, 8, 8, 1.6, 1000.0, -500.0, 4)
    with pytest.raises(gpu_b200.CtrError) as e:
        gpu_b200.Geometry(d)
    assert e.value.status == 8   # CTR_ERR_NO_DEVICE


def test_reference_shim_without_default_geometry():
    import numpy as np
    import gpu_b200
    from gpu_b200 import ctrecon
    if ctrecon.load_library() and getattr(ctrecon, "_default_set", False):
        pytest.skip("default geometry already set in this process")
    v = np.zeros(8, np.float32)
    with pytest.raises(gpu_b200.CtrError):
        gpu_b200.tv_norm_gpu(v)


def _desc_variant(name):
    from gpu_b200 import ctrecon
    base = dict(nx=8, ny=8, nz=8, vx=1.0, nu=8, nv=8, du=1.0, dso=1000.0, dod=-500.0, n_views=4)
    if name == "volume reaches the source":
        return ctrecon.make_desc(**dict(base, vx=200.0))
    if name == "styles exclude each other":
        d = ctrecon.make_desc(**base, ct_style=1)
        d.flags |= ctrecon.GEOM_PARALLEL
        return d
    if name == "tetrahedron beam without sources":
        return ctrecon.make_desc(**base, ct_style=3, n_sources=0)
    if name == "tetrahedron beam with its own z pitch":
        return ctrecon.make_desc(**base, ct_style=3, n_sources=2, vz=2.0)
    if name == "beyond the launch limits":
        return ctrecon.make_desc(**dict(base, nx=70000, vx=0.001))
    if name == "volume beyond 32-bit indices":
        return ctrecon.make_desc(**dict(base, nx=2048, ny=2048, nz=1024, vx=0.1))
    if name == "detector beyond 32-bit indices":
        return ctrecon.make_desc(**dict(base, nu=65536, nv=65536))
    if name == "non-finite angle":
        return ctrecon.make_desc(**base, initial_angle=float("inf"))
    if name == "source at the isocentre":
        return ctrecon.make_desc(**dict(base, dso=0.0))
    if name == "zero detector pitch":
        return ctrecon.make_desc(**dict(base, du=0.0))
    if name == "infinite z pitch":
        return ctrecon.make_desc(**base, vz=float("inf"))
    if name == "voxel pitch below the thresholds' range":
        return ctrecon.make_desc(**dict(base, vx=1e-40))   # 1e-6 of it is below the least float
    raise KeyError(name)


# each rejection and a fragment of its message
REJECTIONS = {
    "volume reaches the source": "reaches the source",
    "styles exclude each other": "exclude each other",
    "tetrahedron beam without sources": "n_sources >= 1",
    "tetrahedron beam with its own z pitch": "single pitches",
    "beyond the launch limits": "launch limits",
    "volume beyond 32-bit indices": "2^31-1",
    "detector beyond 32-bit indices": "detector too large",
    "non-finite angle": "must be finite",
    "source at the isocentre": "0 < dso",
    "zero detector pitch": "pitch must be positive",
    "infinite z pitch": "must be finite",
    "voxel pitch below the thresholds' range": "rounds to 0",
}


@pytest.mark.parametrize("name", sorted(REJECTIONS))
def test_geometry_rejected_before_any_device_call(name):
    """Every rejection of the geometry check returns CTR_ERR_BAD_GEOMETRY with
    a message, before the library touches a device (so it holds on a host
    without a GPU too)."""
    import gpu_b200
    lib = gpu_b200.load_library()
    d = _desc_variant(name)
    h = C.c_void_p()
    assert lib.ctr_geometry_create(C.byref(d), C.byref(h)) == 2      # CTR_ERR_BAD_GEOMETRY
    assert not h.value
    assert REJECTIONS[name] in gpu_b200.last_error()


def test_noalloc_argument_errors_without_device():
    import gpu_b200
    lib = gpu_b200.load_library()
    st = lib.ctr_sart_views_noalloc(None, None, 0, None, 0, C.c_float(0.8), C.c_uint(0), C.c_uint32(0), 0, 1, None)
    assert st == 1                                                   # CTR_ERR_INVALID_ARGUMENT
    assert "NULL" in gpu_b200.last_error()
