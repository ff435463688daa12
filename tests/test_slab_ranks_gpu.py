"""One slab per process (SlabRank, cumc_slab_*): the z-cut grid run as
torch.distributed ranks.  Here the ranks share one GPU, so their process
group is gloo and the ghost planes travel through pinned host buffers (on
several GPUs the same calls go over NCCL); the per-slab C-ABI calls -- the
stage halves, pack and unpack, the seam marks -- and the dt all-reduce are
those of the multi-GPU run.  Against the undivided grid, bit for bit."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cumc3d_b200 import capi, engine, models

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "blast_ring":
        spec, prim, eps = models.blast_3d(24, nx=24, ny=20, nz=24, radius=0.2, p_in=1.0)
        spec["fix_periodic_normal_faces"] = 1
        return spec, prim, eps
    if name == "blast_ring_fp32":
        return models.blast_3d(20, radius=0.2, p_in=1.0, precision="fp32")
    if name == "outflow_weno":
        return models.smooth_state(16, 12, 20, 3, boundary_flag=(0, 0, 1, 1, 1, 1), recon="weno", seed=5)
    if name == "torus_cyl":
        spec, prim, eps = models.torus_cyl(nr=24, nphi=12, nz=24)
        spec["positivity_fallback"] = 1
        return spec, prim, eps
    raise KeyError(name)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, case, sizes, steps, port, out_dir):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        spec, prim, eps = _case(case)
        r = engine.SlabRank(spec, sizes, rank)
        r.set_state(prim, eps)
        r.initial_update()
        dts = []
        for _ in range(steps):
            dt = r.finddt()
            dts.append(dt)
            r.step(dt)
        p, e = r.get_state()
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), p=p, e=e, cons=r.get_array(capi.ARR_CONS),
                 bcell=r.get_array(capi.ARR_BCELL), dts=np.array(dts))
        r.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,sizes,steps", [("blast_ring", (12, 12), 4), ("blast_ring", (8, 9, 7), 3),
                                              ("blast_ring_fp32", (10, 10), 3), ("outflow_weno", (9, 11), 3),
                                              ("torus_cyl", (8, 8, 8), 3)])
def test_ranks_match_the_undivided_grid_bitwise(tmp_path, case, sizes, steps):
    world = len(sizes)
    mp.start_processes(_rank_main, args=(world, case, sizes, steps, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    spec, prim, eps = _case(case)
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    dts = []
    for _ in range(steps):
        dt = s.finddt()
        dts.append(dt)
        s.rungekutta(dt)
    parts = [np.load(tmp_path / ("r%d.npz" % r)) for r in range(world)]
    for p in parts:
        assert np.array_equal(p["dts"], np.array(dts))
    nz = spec["nz"]
    ps, es = s.get_state()
    want = {"p": ps[3:nz + 3], "e": es[3:nz + 3], "cons": s.get_array(capi.ARR_CONS)[3:nz + 3],
            "bcell": s.get_array(capi.ARR_BCELL)[3:nz + 3]}
    for k, b in want.items():
        a = np.concatenate([p[k] for p in parts], axis=0)[:, 3:-3, 3:-3]
        b = b[:, 3:-3, 3:-3]
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (k, int((a != b).sum()))
    s.close()


def test_slab_calls_refuse_what_a_slab_cannot_do():
    import ctypes
    spec, prim, eps = models.blast_3d(12)
    nb = ctypes.c_size_t()
    s = engine.Solver(spec)   # not a slab: no exchanged side
    assert s.L.cumc_slab_halo_bytes(s.h, engine.FILL_STATE, 0, ctypes.byref(nb)) == capi.CUMC_EINVAL
    assert s.L.cumc_slab_initial_begin(s.h) == capi.CUMC_EINVAL
    s.close()
    specs, _ = engine.slab_specs(spec, (6, 6))
    a = engine.Solver(specs[0])
    L, h = a.L, a.h
    assert L.cumc_slab_halo_bytes(h, 2, 0, ctypes.byref(nb)) == capi.CUMC_EINVAL                # no such fill
    assert L.cumc_slab_halo_bytes(h, engine.FILL_EMF, 2, ctypes.byref(nb)) == capi.CUMC_EINVAL  # no such side
    assert L.cumc_slab_stage(h, 1, 0) == capi.CUMC_ENOTREADY          # before INITIAL_UPDATE
    a.set_state(prim[:12], eps[:12])
    assert L.cumc_slab_initial_begin(h) == 0 and L.cumc_slab_initial_end(h) == 0
    assert L.cumc_slab_seam(h, 0) == capi.CUMC_EINVAL                 # too late to mark the seam
    assert L.cumc_slab_step_begin(h, -1.0) == capi.CUMC_EINVAL
    assert L.cumc_slab_stage(h, 4, 0) == capi.CUMC_EINVAL
    a.close()
