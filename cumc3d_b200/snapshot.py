"""Output snapshots: the datasets of the reference's print_hydroprofile
(solver/mhd/dataio.f90:31-240, file ``rkiter-<n>-nm.hdf5``): time,
dimension, coordinate (coordinate_flag + 1), x/y/z-interface (faces -1..n+1),
primitive (prim(1:5, 0:n+1, ...)), epsilon (0:n+1 each axis), bfield
(prim(ibx:ibz, -1:n+1, ...)).

The engine fills the three state arrays on the device and copies them out
on a separate stream (``Solver.snapshot_start`` / ``snapshot_wait``), so the
step loop does not wait for the output.  HDF5 has no Python binding on this
image, so ``write`` stores the same datasets, under the same names, in an
``.npz`` container; each array's C-order shape is the Fortran shape reversed,
which is also what an HDF5 reader shows for the reference's files, so a
converter only has to copy arrays across.
"""
import numpy as np


def buffers(spec, pinned=False):
    """(primitive, epsilon, bfield) arrays for one snapshot.  pinned=True
    allocates page-locked host memory (through torch), which lets the copy
    overlap the following steps."""
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    shapes = ((nz + 2, ny + 2, nx + 2, 5), (nz + 2, ny + 2, nx + 2), (nz + 3, ny + 3, nx + 3, 3))
    if pinned:
        import torch
        return tuple(torch.empty(s, dtype=torch.float64).pin_memory().numpy() for s in shapes)
    return tuple(np.empty(s) for s in shapes)


def write(path, spec, time, primitive, epsilon, bfield):
    """One snapshot file with the reference's dataset names."""
    np.savez(path, **{
        "time": np.array([time]),
        "dimension": np.array([float(spec["n_dim"])]),
        "coordinate": np.array([float(spec.get("coordinate_flag", 0) + 1)]),
        "x-interface": np.asarray(spec["xF"])[2:spec["nx"] + 5],
        "y-interface": np.asarray(spec["yF"])[2:spec["ny"] + 5],
        "z-interface": np.asarray(spec["zF"])[2:spec["nz"] + 5],
        "primitive": primitive, "epsilon": epsilon, "bfield": bfield,
    })


def read(path):
    """dict of the datasets of a snapshot file."""
    with np.load(path) as f:
        return {k: f[k] for k in f.files}
