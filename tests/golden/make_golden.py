"""Generate tests/golden/*.npz from the reference's own kernels.

Runs the reference's CUDA kernel sources compiled for the CPU
(oracle/_ref/libctref*.so, one per CT_style, built by
`make -C oracle REF_ROOT=<reference checkout>`) on seeded inputs for the small scans of
tests/scan_configs.py (cone beam, and the fan-slice and parallel geometries)
and the tetrahedron-beam program's (libctref_tbct.so), and stores inputs
and outputs.  The fixtures pin the C restatement in
oracle/ct_oracle.c where the reference checkout is absent.

    python tests/golden/make_golden.py [scan names ...]   (default: all)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import ctoracle  # noqa: E402
from scan_configs import SMALL, STYLES, TBCT, og_desc  # noqa: E402


def main():
    ctoracle.build()
    only = set(sys.argv[1:])
    for name, cfg in list(SMALL.items()) + list(STYLES.items()) + list(TBCT.items()):
        if only and name not in only:
            continue
        cone = cfg.get("ct_style", 0) == 0
        # the tetrahedron-beam program: projector, backprojection + update and
        # its SART pass only (its backprojector has no command 0; its FGP is
        # the cone-beam program's, pinned above)
        tbct = cfg.get("ct_style", 0) == 3
        if cfg["nx"] != cfg["ny"] or cfg["ny"] != cfg["nz"]:
            d = og_desc(cfg)
            d.nx, d.ny, d.nz = cfg["nx"], cfg["ny"], cfg["nz"]
        else:
            d = og_desc(cfg)
        ref = ctoracle.RefOracle(d)
        rng = np.random.default_rng(1234)
        vol = rng.uniform(0.0, 0.05, ref.vol_shape).astype(np.float32)
        nv = cfg["nviews"]
        fp0 = np.stack([ref.forward_view(vol, j, 0) for j in range(nv)])
        b = (fp0 * (1.0 + 0.01 * rng.standard_normal(fp0.shape))).astype(np.float32)
        fp1 = np.stack([ref.forward_view(vol, j, 1, b[j]) for j in range(nv)])
        bpv = [0, nv // 3, nv - 1]
        corr = rng.standard_normal((len(bpv),) + ref.view_shape).astype(np.float32)
        bp1 = np.stack([ref.backproject_view(vol, corr[a], j, 0.8, 1) for a, j in enumerate(bpv)])
        sart = ref.sart(np.zeros_like(vol), b, 0.8)
        if tbct:
            bp0 = fgp = np.zeros(0, np.float32)
            tv = l2 = 0.0
        else:
            bp0 = np.stack([ref.backproject_view(np.zeros_like(vol), corr[a], j, 1.0, 0) for a, j in enumerate(bpv)])
            fgp = ref.fgp(vol, 0.01, 5)
            tv = ref.tv_norm(vol)
            l2 = ref.l2_norm(fp0, b)
        fdkw = ramp = fdkbp = np.zeros(0, np.float32)   # FDK is the cone beam's only
        if cone:
            fdkw = ref.fdk_weight(b)
            ramp = ref.ramp_filter(fdkw[:2])
            fdkbp = np.zeros_like(vol)
            for j in range(min(nv, 4)):
                fdkbp = ref.fdk_bp_view(fdkbp, ramp[0] if j % 2 == 0 else ramp[1], j)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            vol=vol, b=b, fp0=fp0, fp1=fp1, bp_views=np.array(bpv), corr=corr, bp1=bp1, bp0=bp0, sart=sart,
            fgp=fgp, fgp_lambda=np.float32(0.01), fgp_iters=np.int32(5), tv=np.float64(tv), l2=np.float64(l2),
            fdkw=fdkw, ramp=ramp, fdkbp=fdkbp,
        )
        print(name, "written")


if __name__ == "__main__":
    main()
