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
import json

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


DATASETS = ("time", "dimension", "coordinate", "x-interface", "y-interface", "z-interface", "primitive", "epsilon",
            "bfield")


def write_raw(prefix, spec, time, primitive, epsilon, bfield):
    """The same datasets as raw little-endian FP64 files ``<prefix>.<name>.bin``
    plus ``<prefix>.json`` (each dataset's Fortran shape and byte order).  A C
    array whose shape is the Fortran shape reversed has the Fortran array's
    memory layout, so each file is also the bytes of the reference's array
    in its own order (dataio.f90 passes prim(imin:ibx-1,0:nx+1,...) etc.)."""
    data = dict(np.load(_npz_bytes(spec, time, primitive, epsilon, bfield)))
    manifest = {}
    for name in DATASETS:
        a = np.ascontiguousarray(data[name], dtype="<f8")
        with open("%s.%s.bin" % (prefix, name), "wb") as f:
            f.write(a.tobytes())
        manifest[name] = {"fortran_shape": list(a.shape[::-1]), "c_shape": list(a.shape), "dtype": "<f8"}
    with open(prefix + ".json", "w") as f:
        json.dump(manifest, f, indent=1)
    return manifest


def _npz_bytes(spec, time, primitive, epsilon, bfield):
    import io
    buf = io.BytesIO()
    write(buf, spec, time, primitive, epsilon, bfield)
    buf.seek(0)
    return buf


def read_raw(prefix):
    """dict of the datasets of a raw snapshot (C-order arrays)."""
    with open(prefix + ".json") as f:
        manifest = json.load(f)
    return {name: np.fromfile("%s.%s.bin" % (prefix, name), dtype=m["dtype"]).reshape(m["c_shape"])
            for name, m in manifest.items()}


def to_hdf5(source, h5path):
    """Convert a snapshot (an ``.npz`` from ``write`` or the prefix of a raw
    snapshot) to an HDF5 file with the reference's dataset names and shapes
    (``rkiter-<n>-nm.hdf5`` of dataio.f90:31-240).  Needs h5py, which this
    image does not have; the datasets are written as they are (their C
    shapes are what an HDF5 reader shows for the reference's own files)."""
    try:
        import h5py
    except ImportError as ex:
        raise RuntimeError("to_hdf5 needs h5py (not installed here); the .npz and raw snapshots carry the same "
                           "datasets") from ex
    data = read(source) if str(source).endswith(".npz") else read_raw(source)
    with h5py.File(h5path, "w") as f:
        for name in DATASETS:
            f.create_dataset(name, data=np.asarray(data[name], dtype=np.float64))
    return h5path
