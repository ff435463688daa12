"""ctypes mirror of include/cumc3d_gpu.h (structures and constants only).

The structures here are the host-side image of ``cumc_config`` and
``cumc_model``; the same structures are handed to the CUDA library
(:mod:`cumc3d_b200.engine`).  Field order and types must match the header.
"""
import ctypes as C

import numpy as np

# status codes
CUMC_OK = 0
CUMC_EINVAL = 1
CUMC_ECUDA = 2
CUMC_ENOMEM = 3
CUMC_ESTATE = 4
CUMC_ENOTREADY = 5

# reconstruction (solver/mhd/parameter.h:102-115)
RECON = {"tvdmm": 0, "tvdvl": 1, "tvdmc": 2, "ppm": 3, "weno": 4}
# Riemann solvers (solver/mhd/parameter.h:90-100)
RIEMANN = {"lf": 0, "hll": 1, "hllc": 2, "hlld": 3}
PRECISION = {"fp64": 0, "fp32": 1}
BOUNDARY_EXCHANGE = 9  # boundary_flag of a z side shared with a neighbouring slab
FLOOR = {"none": 0, "eps": 1, "torus": 2, "collapsar": 3}
SOURCE = {"none": 0, "const_gy": 1, "pm_cyl": 2, "pm_sph": 3, "collapsar": 4}
BCHOOK = {"none": 0, "torus_cyl": 1, "torus_sph": 2}

ARR_CONS = 0
ARR_BCELL = 1
ARR_CS = 2

# variable order of prim/cons (solver/mhd/setup.f90:39-90), 0-based here
IRHO, IVX, IVY, IVZ, ITAU, IBX, IBY, IBZ = range(8)


class CumcModel(C.Structure):
    _fields_ = [
        ("gamma", C.c_double),
        ("floor_kind", C.c_int),
        ("rho_floor", C.c_double),
        ("eps_floor", C.c_double),
        ("p_floor", C.c_double),
        ("source_kind", C.c_int),
        ("g_const", C.c_double),
        ("r_sh", C.c_double),
        ("bc_kind", C.c_int),
    ]


class CumcConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("n_dim", C.c_int),
        ("coordinate_flag", C.c_int),
        ("boundary_flag", C.c_int * 6),
        ("xF", C.POINTER(C.c_double)),
        ("yF", C.POINTER(C.c_double)),
        ("zF", C.POINTER(C.c_double)),
        ("cfl", C.c_double),
        ("recon", C.c_int),
        ("riemann", C.c_int),
        ("precision", C.c_int),
        ("learned", C.c_int),
        ("fixpole", C.c_int),
        ("fix_periodic_normal_faces", C.c_int),
        ("positivity_fallback", C.c_int),
        ("model", CumcModel),
    ]


class CumcBatchConfig(C.Structure):
    _fields_ = [
        ("n_problems", C.c_int),
        ("nx", C.POINTER(C.c_int)),
        ("xF", C.POINTER(C.POINTER(C.c_double))),
        ("t_end", C.POINTER(C.c_double)),
        ("cfl", C.c_double), ("gamma", C.c_double),
        ("recon", C.c_int), ("riemann", C.c_int), ("precision", C.c_int),
        ("floor_kind", C.c_int),
        ("positivity_fallback", C.c_int),
    ]


class CumcTrainConfig(C.Structure):
    _fields_ = [
        ("steps", C.c_int), ("batch", C.c_int),
        ("lr", C.c_float), ("delta", C.c_float),
        ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
        ("seed", C.c_ulonglong),
    ]


LEARN_NP, LEARN_NF, LEARN_ROW = 2657, 35, 37


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# the keys of a spec's "model" dict (the fields of cumc_model)
MODEL_KEYS = {"gamma", "floor", "rho_floor", "eps_floor", "p_floor", "source", "g_const", "r_sh", "bc"}


def make_config(spec):
    """Build a ``CumcConfig`` from a plain dict (see :mod:`cumc3d_b200.models`).

    Returns ``(config, keepalive)``; keep ``keepalive`` referenced while the
    config is in use, it owns the face-coordinate arrays.
    """
    xF = np.ascontiguousarray(spec["xF"], dtype=np.float64)
    yF = np.ascontiguousarray(spec["yF"], dtype=np.float64)
    zF = np.ascontiguousarray(spec["zF"], dtype=np.float64)
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    if xF.size != nx + 7 or yF.size != ny + 7 or zF.size != nz + 7:
        raise ValueError("face arrays must hold indices -3..n+3")
    m = spec.get("model", {})
    unknown = sorted(set(m) - MODEL_KEYS)
    if unknown:
        raise ValueError("unknown model descriptor keys: %s" % ", ".join(unknown))
    model = CumcModel(
        gamma=float(m.get("gamma", 5.0 / 3.0)),
        floor_kind=FLOOR[m.get("floor", "none")],
        rho_floor=float(m.get("rho_floor", 0.0)),
        eps_floor=float(m.get("eps_floor", 0.0)),
        p_floor=float(m.get("p_floor", 0.0)),
        source_kind=SOURCE[m.get("source", "none")],
        g_const=float(m.get("g_const", 0.1)),
        r_sh=float(m.get("r_sh", 0.0)),
        bc_kind=BCHOOK[m.get("bc", "none")],
    )
    cfg = CumcConfig()
    cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
    cfg.n_dim = spec["n_dim"]
    cfg.coordinate_flag = spec.get("coordinate_flag", 0)
    for i, b in enumerate(spec["boundary_flag"]):
        cfg.boundary_flag[i] = b
    cfg.xF, cfg.yF, cfg.zF = _dptr(xF), _dptr(yF), _dptr(zF)
    cfg.cfl = float(spec["cfl"])
    cfg.recon = RECON[spec["recon"]]
    cfg.riemann = RIEMANN[spec["riemann"]]
    cfg.precision = PRECISION[spec.get("precision", "fp64")]
    cfg.learned = int(spec.get("learned", 0))
    cfg.fixpole = int(spec.get("fixpole", 0))
    cfg.fix_periodic_normal_faces = int(spec.get("fix_periodic_normal_faces", 0))
    cfg.positivity_fallback = int(spec.get("positivity_fallback", 0))
    cfg.model = model
    return cfg, (xF, yF, zF)


def padded_shape(spec):
    """numpy shape of prim in the Fortran layout: (nz+6, ny+6, nx+6, 8)."""
    return (spec["nz"] + 6, spec["ny"] + 6, spec["nx"] + 6, 8)
