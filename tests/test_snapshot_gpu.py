"""Output snapshots (cumc_snapshot_start / wait): the reference's output
datasets (solver/mhd/dataio.f90:31-240) packed on the device and copied out
on a separate stream while later steps run; the snapshot holds the state as
of its start, bit for bit."""
import numpy as np
import pytest

from cumc3d_b200 import engine, models, snapshot

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pinned", [True, False])
def test_snapshot_is_the_state_at_its_start(pinned, tmp_path):
    spec, prim, eps = models.blast_3d(20, nx=20, ny=16, nz=12, radius=0.2, p_in=1.0)
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    for _ in range(2):
        s.rungekutta(s.finddt())
    p0, e0 = s.get_state()
    bufs = snapshot.buffers(spec, pinned=pinned)
    s.snapshot_start(*bufs)
    for _ in range(3):  # these steps run while the copy is in flight
        s.rungekutta(s.finddt())
    s.snapshot_wait()
    primitive, epsilon, bfield = bufs
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    # padded arrays hold cells -2..n+3 at index j + 2
    assert np.array_equal(primitive.view(np.uint64), p0[2:nz + 4, 2:ny + 4, 2:nx + 4, 0:5].view(np.uint64))
    assert np.array_equal(epsilon.view(np.uint64), e0[2:nz + 4, 2:ny + 4, 2:nx + 4].view(np.uint64))
    assert np.array_equal(bfield.view(np.uint64), p0[1:nz + 4, 1:ny + 4, 1:nx + 4, 5:8].view(np.uint64))
    p1, _ = s.get_state()
    assert not np.array_equal(p1, p0)  # the later steps did change the state
    path = tmp_path / "rkiter-2-nm.npz"
    snapshot.write(path, spec, 0.0, primitive, epsilon, bfield)
    back = snapshot.read(path)
    assert np.array_equal(back["primitive"], primitive) and np.array_equal(back["bfield"], bfield)
    s.close()


def test_a_second_snapshot_waits_for_the_first():
    spec, prim, eps = models.blast_3d(12, radius=0.2, p_in=1.0)
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    a, b = snapshot.buffers(spec, pinned=True), snapshot.buffers(spec, pinned=True)
    s.snapshot_start(*a)
    s.rungekutta(s.finddt())
    s.snapshot_start(*b)  # waits for a, then copies the stepped state
    s.snapshot_wait()
    assert not np.array_equal(a[0], b[0])
    p, e = s.get_state()
    n = 12
    assert np.array_equal(b[1], e[2:n + 4, 2:n + 4, 2:n + 4])
    s.close()
