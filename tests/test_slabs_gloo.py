"""The one-slab-per-rank driver (gpu_b200/slabs.py) as gloo ranks on the CPU.

Each rank holds its z-slab of the volume and runs SlabSART: its slab's
partial sums, the all-gather of every rank's parts, the combination in rank
order, its slab's update.  The per-view steps are CPU stand-ins built from
the oracle (the GPU library's ctr_forward_partial / ctr_combine_partials /
ctr_sart_update are checked against the same oracle functions in
tests/test_gpu_slabs.py), so what runs here is the driver's exchange and
ordering.  The slabs the ranks end with must equal the reference's D-device
pass (golden fixtures from its multi-GPU kernels) and, with the engine's
update, the oracle's D-slab pass.  Rendezvous on 127.0.0.1.
"""
import json
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleSlabOps:
    """CPU stand-ins for the three per-view steps of one slab."""

    def __init__(self, co, desc, n_slabs, slab, engine):
        self.o = co.Oracle(co.slab_desc(desc, n_slabs, slab))
        self.engine = engine

    @property
    def view_shape(self):
        return self.o.view_shape

    def forward_partial(self, vol, view, part, tiled=False):
        import torch
        w, ln = self.o.forward_partial(vol.numpy(), view)
        part[..., 0] = torch.from_numpy(w)
        part[..., 1] = torch.from_numpy(ln)

    def combine(self, parts, view, b_view, rays):
        import torch
        p = parts.numpy()
        rays[..., 0] = torch.from_numpy(self.o.combine_partials(p[..., 0].copy(), p[..., 1].copy(), b_view.numpy()))
        rays[..., 1] = 0.0

    def update(self, vol, rays, view, beta, flags=0, seed=0, tiled=False):
        import torch
        c = np.ascontiguousarray(rays[..., 0].numpy())
        out = (self.o.backproject_gather(vol.numpy(), c, view, beta) if self.engine
               else self.o.backproject_ref(vol.numpy(), c, view, beta, 1))
        vol.copy_(torch.from_numpy(out))


def _rank_main(rank, world, port, name, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from gpu_b200.slabs import SlabSART, slab_of
    from oracle import ctoracle as co
    from scan_configs import SLABS, og_desc

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    cfg = SLABS[name]
    g = dict(np.load(os.path.join(HERE, "golden", f"slabs_{name}.npz")))
    sino = torch.from_numpy(g["b"])
    res = {}
    for engine in (False, True):
        ops = OracleSlabOps(co, og_desc(cfg), world, rank, engine)
        vol = slab_of(torch.from_numpy(g["vol0"]), rank, world).clone()
        SlabSART(ops, rank, world, "cpu").views(vol, sino, 0.8, 0, cfg["nviews"])
        np.save(os.path.join(out_dir, f"{'engine' if engine else 'ref'}_{rank}.npy"), vol.numpy())
        res[engine] = True
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"done_{rank}.json"), "w") as f:
        json.dump({"rank": rank}, f)


@pytest.mark.parametrize("name,world", [("cube16", 2), ("cone_wide", 4)])
def test_ranks_reproduce_the_multi_device_pass(name, world, tmp_path, oracle_built):
    mp = pytest.importorskip("torch.multiprocessing")
    oracle_built.build()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, name, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    from scan_configs import SLABS, og_desc
    g = dict(np.load(os.path.join(HERE, "golden", f"slabs_{name}.npz")))
    ref = np.concatenate([np.load(tmp_path / f"ref_{r}.npy") for r in range(world)])
    np.testing.assert_array_equal(ref.view(np.uint32), g[f"sart_{world}"].view(np.uint32))
    eng = np.concatenate([np.load(tmp_path / f"engine_{r}.npy") for r in range(world)])
    o = oracle_built.Oracle(og_desc(SLABS[name]))
    want = o.sart_pass_slabs(g["vol0"], g["b"], 0.8, world, engine=True)
    np.testing.assert_array_equal(eng.view(np.uint32), want.view(np.uint32))
