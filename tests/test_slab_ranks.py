"""One slab per rank (CPU: gloo, world sizes 2-4): the halo protocol that
SlabRank runs at every exchange point -- which neighbour each side talks
to, and the order of the point-to-point messages, including a ring of two
slabs whose both neighbours are the same rank.  The slabs here are numpy
stand-ins with the engine's plane layout (padded planes -2..m+3; side 0
packs planes 1..3 and unpacks into -2..0, side 1 packs m-2..m and unpacks
into m+1..m+3) and the engine's uneven buffer sizes (a cut inside the grid
carries one array more than the periodic seam)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cumc3d_b200 import engine

NV = 4       # values per plane
SIZES = [4, 3, 5, 4]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_neighbours_of_a_ring_and_of_a_bounded_axis():
    assert [engine.halo_peers(r, 3, True) for r in range(3)] == [(2, 1), (0, 2), (1, 0)]
    assert [engine.halo_peers(r, 3, False) for r in range(3)] == [(None, 1), (0, 2), (1, None)]
    assert [engine.halo_peers(r, 2, True) for r in range(2)] == [(1, 1), (0, 0)]


class FakeSlab:
    """Planes (m+6, arrays, NV) with global cell numbers in the interior."""

    def __init__(self, rank, world, ring):
        self.m, self.offset = SIZES[rank], sum(SIZES[:rank])
        self.peers = engine.halo_peers(rank, world, ring)
        self.seam = (ring and rank == 0, ring and rank == world - 1)
        self.a = np.full((self.m + 6, 9, NV), np.nan)
        for l in range(1, self.m + 1):
            self.a[l + 2] = (self.offset + l) + 0.01 * np.arange(9)[:, None] + 1e-4 * np.arange(NV)[None, :]

    def arrays(self, fill, side):
        # the state fill of a cut inside the grid carries one array more
        return (9 if not self.seam[side] else 8) if fill == engine.FILL_STATE else 7

    def pack(self, fill, side):
        m = self.m
        rows = slice(3, 6) if side == 0 else slice(m, m + 3)
        return torch.from_numpy(np.ascontiguousarray(self.a[rows, :self.arrays(fill, side)].transpose(1, 0, 2)).ravel())

    def unpack(self, fill, side, buf):
        m, k = self.m, self.arrays(fill, side)
        rows = slice(0, 3) if side == 0 else slice(m + 3, m + 6)
        self.a[rows, :k] = buf.numpy().reshape(k, 3, NV).transpose(1, 0, 2)


def _rank_main(rank, world, ring, tags, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        s = FakeSlab(rank, world, ring)
        for fill in (engine.FILL_EMF, engine.FILL_STATE):
            sides = [d for d in (0, 1) if s.peers[d] is not None]
            send = {d: s.pack(fill, d) for d in sides}
            recv = {d: torch.empty_like(send[d]) for d in sides}
            for w in dist.batch_isend_irecv(engine.halo_p2p_ops(s.peers, send, recv, tags=tags)):
                w.wait()
            for d in sides:
                s.unpack(fill, d, recv[d])
        np.save(os.path.join(out_dir, "r%d.npy" % rank), s.a)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,ring,tags", [(2, True, True), (2, True, False), (3, True, False), (4, True, True),
                                             (2, False, True), (3, False, False)])
def test_ghost_planes_hold_the_neighbours_cells(tmp_path, world, ring, tags):
    """tags=False: messages matched by posting order alone, as NCCL does."""
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, ring, tags, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    nz = sum(SIZES[:world])
    for r in range(world):
        a = np.load(tmp_path / ("r%d.npy" % r))
        m, off = SIZES[r], sum(SIZES[:r])
        for side, ls in ((0, range(-2, 1)), (1, range(m + 1, m + 4))):
            seam = ring and ((side == 0 and r == 0) or (side == 1 and r == world - 1))
            bounded = not ring and ((side == 0 and r == 0) or (side == 1 and r == world - 1))
            for l in ls:
                g = off + l
                if bounded:
                    assert np.all(np.isnan(a[l + 2]))
                    continue
                g = (g - 1) % nz + 1
                k = 8 if seam else 9
                want = g + 0.01 * np.arange(k)[:, None] + 1e-4 * np.arange(NV)[None, :]
                assert np.array_equal(a[l + 2, :k], want), (r, side, l)


def _leaving_rank_main(rank, world, port, out_dir):
    import datetime
    import time
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    try:
        s = FakeSlab(rank, world, False)
        dist.barrier()                      # one step together
        if rank == 1:
            return                          # leaves between steps, nothing in flight
        sides = [d for d in (0, 1) if s.peers[d] is not None]
        send = {d: s.pack(engine.FILL_STATE, d) for d in sides}
        recv = {d: torch.empty_like(send[d]) for d in sides}
        t0 = time.time()
        try:
            for w in dist.batch_isend_irecv(engine.halo_p2p_ops(s.peers, send, recv)):
                w.wait()
            outcome = "completed"
        except RuntimeError:
            outcome = "error"
        with open(os.path.join(out_dir, "r0.txt"), "w") as f:
            f.write("%s %.1f" % (outcome, time.time() - t0))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_a_rank_that_leaves_ends_its_neighbours_exchange_with_an_error(tmp_path):
    """Failure detection on the host: rank 1 leaves between steps; rank 0's
    next halo exchange ends with an error (the peer's connection closes, or
    the process group's 5 s timeout runs out) instead of waiting for good."""
    mp.start_processes(_leaving_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    outcome, secs = (tmp_path / "r0.txt").read_text().split()
    assert outcome == "error" and float(secs) < 60
