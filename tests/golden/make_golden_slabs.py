"""Generate tests/golden/slabs_*.npz from the reference's multi-GPU kernels.

Runs V63/kernel_IterativeRecon_universal_multiGPU.cu compiled for the CPU
(oracle/_ref/libctref*.so, through oracle/ref_harness.cpp) with the host
sequence of V63/host_IterativeRecon_CBCT_multiGPU.c, the devices becoming a
loop over the slabs -- for the tetrahedron-beam scans the program's own
multi-GPU build (T42/voxel/*_multiGPU.*, oracle/_ref/libctref_tbct_multi.so)
-- for the scans of scan_configs.SLABS and each of their slab counts D.
Stored per scan: the seeded start volume (with -0 planted), the sinogram,
and per D the whole SART pass from that volume, one view's partial sums and
correction, that view's slab backprojections (commands 0 and 1; the
tetrahedron beam's kernels have no command) and the D-device build's
row-split forward projection of the start volume at that view.  The
fixtures pin oracle/ct_oracle.c's slab functions where the reference
checkout is absent.

    python tests/golden/make_golden_slabs.py [scan names ...]   (default: all)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import ctoracle  # noqa: E402
from scan_configs import SLABS, og_desc  # noqa: E402

VIEW = 1   # the view whose pieces are stored


def main():
    ctoracle.build()
    only = set(sys.argv[1:])
    for name, cfg in SLABS.items():
        if only and name not in only:
            continue
        d = og_desc(cfg)
        one = ctoracle.RefOracle(d)                                   # the one-device build
        ref = ctoracle.RefOracle(d, multi=True)                       # its multi-GPU kernels
        rng = np.random.default_rng(4321)
        truth = rng.uniform(0.0, 0.05, one.vol_shape).astype(np.float32)
        nv = cfg["nviews"]
        b = np.stack([one.forward_view(truth, j, 0) for j in range(nv)]).astype(np.float32)
        vol0 = rng.uniform(0.0, 0.03, one.vol_shape).astype(np.float32)
        vol0[rng.uniform(size=vol0.shape) < 0.1] = -0.0
        out = dict(b=b, vol0=vol0, slabs=np.array(cfg["slabs"], np.int32), view=np.int32(VIEW))
        for D in cfg["slabs"]:
            zs = cfg["nz"] // D
            # the row-split forward of the D-device build: for V63 the one-device forward
            if cfg.get("ct_style", 0) != 3:
                for j in range(nv):
                    a, c = ref.forward_view_split(truth, D, j), one.forward_view(truth, j, 0)
                    assert np.array_equal(a.view(np.uint32), c.view(np.uint32)), (name, D, j)
            out[f"fwd_split_{D}"] = ref.forward_view_split(vol0, D, VIEW)
            out[f"sart_{D}"] = ref.sart_slabs(vol0, b, 0.8, D)
            parts = [ref.slab_forward_view(vol0[zs * s:zs * (s + 1)], D, s, VIEW) for s in range(D)]
            w = np.stack([p[0] for p in parts])
            ln = np.stack([p[1] for p in parts])
            corr = ref.combine_view(w, ln, b[VIEW])
            out[f"w_{D}"], out[f"l_{D}"], out[f"corr_{D}"] = w, ln, corr
            out[f"bp1_{D}"] = np.concatenate([ref.slab_backproject_view(vol0[zs * s:zs * (s + 1)], corr, D, s, VIEW,
                                                                        0.8, 1) for s in range(D)])
            out[f"bp0_{D}"] = np.concatenate([ref.slab_backproject_view(np.zeros_like(vol0[zs * s:zs * (s + 1)]),
                                                                        corr, D, s, VIEW, 1.0, 0) for s in range(D)])
        np.savez_compressed(os.path.join(HERE, f"slabs_{name}.npz"), **out)
        print("wrote", name, cfg["slabs"])


if __name__ == "__main__":
    main()
