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
