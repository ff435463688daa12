"""Host-side driver of the B200 engine, over the C-ABI in include/cumc3d_gpu.h.

:class:`Solver` mirrors the reference's time loop (solver/mhd/main.f90:50-139)
and keeps its routine names: ``initial_update`` (INITIAL_UPDATE), ``finddt``
(FINDDT), ``rungekutta`` (RUNGEKUTTA), ``find_divb`` (FIND_DIVB).  Every call
goes through ``libcumc3d_gpu.so``; there is no CPU path.  A missing library or
a missing CUDA device raises immediately.
"""
import ctypes as C
import os

import numpy as np

from . import capi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcumc3d_gpu.so")

# every symbol include/cumc3d_gpu.h declares
EXPORTS = [
    "cumc_create", "cumc_destroy", "cumc_set_state", "cumc_get_state", "cumc_get_array",
    "cumc_initial_update", "cumc_finddt", "cumc_rk3_step", "cumc_evolve", "cumc_max_divb",
    "cumc_sync", "cumc_launch_count", "cumc_stream", "cumc_profile_step", "cumc_fp64_peak", "cumc_autotune",
    "cumc_set_tuning", "cumc_set_concurrent_sweeps", "cumc_fallback_count", "cumc_check_div3", "cumc_check_dv",
    "cumc_batch_create", "cumc_batch_destroy", "cumc_batch_set_state", "cumc_batch_get_state",
    "cumc_batch_run", "cumc_batch_sync", "cumc_batch_stream", "cumc_batch_launch_count", "cumc_batch_last_error",
    "cumc_batch_set_cluster",
    "cumc_batch_run1_noalloc",
    "cumc_learn_set", "cumc_learn_stats", "cumc_learn_flags", "cumc_learn_harvest",
    "cumc_poisson_setup", "cumc_poisson_solve", "cumc_poisson_get", "cumc_poisson_set",
    "cumc_collapsar_set", "cumc_collapsar_get", "cumc_snapshot_start", "cumc_snapshot_wait",
    "cumc_group_initial_update", "cumc_group_finddt", "cumc_group_step",
    "cumc_slab_seam", "cumc_slab_halo_bytes", "cumc_slab_halo_pack", "cumc_slab_halo_unpack",
    "cumc_slab_initial_begin", "cumc_slab_initial_end", "cumc_slab_step_begin", "cumc_slab_stage",
    "cumc_slab_step_end", "cumc_mlp_grad", "cumc_mlp_train",
    "cumc_mlp_infer", "cumc_mlp_last_error",
    "cumc_last_error",
]

PROFILE_CLASSES = ["flux_x", "flux_y", "flux_z", "emf", "rk", "recover", "boundary", "dt"]

_lib = None


class CumcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cumc error %d: %s" % (code, msg))
        self.code = code


def load_library(path=None):
    """Load the CUDA engine; raises if the shared library is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("CUDA engine library missing: %s (run python -m cumc3d_b200.build)" % p)
    L = C.CDLL(p)
    L.cumc_create.argtypes = [C.POINTER(capi.CumcConfig), C.POINTER(C.c_void_p)]
    L.cumc_destroy.argtypes = [C.c_void_p]
    L.cumc_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.cumc_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.cumc_get_array.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    L.cumc_initial_update.argtypes = [C.c_void_p]
    L.cumc_finddt.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.cumc_rk3_step.argtypes = [C.c_void_p, C.c_double]
    L.cumc_evolve.argtypes = [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.cumc_max_divb.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.cumc_sync.argtypes = [C.c_void_p]
    L.cumc_launch_count.argtypes = [C.c_void_p]
    L.cumc_launch_count.restype = C.c_int64
    L.cumc_stream.argtypes = [C.c_void_p]
    L.cumc_stream.restype = C.c_void_p
    L.cumc_profile_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int]
    L.cumc_fp64_peak.argtypes = [C.POINTER(C.c_double)]
    L.cumc_autotune.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.cumc_set_tuning.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.cumc_set_concurrent_sweeps.argtypes = [C.c_void_p, C.c_int]
    L.cumc_fallback_count.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_ulonglong)]
    L.cumc_check_div3.argtypes = [C.c_ulonglong, C.c_longlong, C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)]
    L.cumc_check_dv.argtypes = [C.c_ulonglong, C.c_longlong, C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)]
    L.cumc_last_error.argtypes = [C.c_void_p]
    L.cumc_last_error.restype = C.c_char_p
    L.cumc_batch_create.argtypes = [C.POINTER(capi.CumcBatchConfig), C.POINTER(C.c_void_p)]
    L.cumc_batch_destroy.argtypes = [C.c_void_p]
    L.cumc_batch_set_state.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.cumc_batch_get_state.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.cumc_batch_run.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.cumc_batch_sync.argtypes = [C.c_void_p]
    L.cumc_batch_stream.argtypes = [C.c_void_p]
    L.cumc_batch_stream.restype = C.c_void_p
    L.cumc_batch_launch_count.argtypes = [C.c_void_p]
    L.cumc_batch_set_cluster.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.cumc_batch_launch_count.restype = C.c_int64
    L.cumc_batch_last_error.argtypes = [C.c_void_p]
    L.cumc_batch_last_error.restype = C.c_char_p
    L.cumc_learn_set.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_float]
    L.cumc_learn_stats.argtypes = [C.c_void_p, C.c_void_p]
    L.cumc_poisson_setup.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.cumc_poisson_solve.argtypes = [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.POINTER(C.c_int)]
    L.cumc_poisson_get.argtypes = [C.c_void_p, C.c_void_p]
    L.cumc_poisson_set.argtypes = [C.c_void_p, C.c_void_p]
    L.cumc_collapsar_set.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.cumc_snapshot_start.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.cumc_snapshot_wait.argtypes = [C.c_void_p]
    L.cumc_group_initial_update.argtypes = [C.c_void_p, C.c_int]
    L.cumc_group_finddt.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    L.cumc_group_step.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.cumc_slab_seam.argtypes = [C.c_void_p, C.c_int]
    L.cumc_slab_halo_bytes.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_size_t)]
    L.cumc_slab_halo_pack.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.cumc_slab_halo_unpack.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.cumc_slab_initial_begin.argtypes = [C.c_void_p]
    L.cumc_slab_initial_end.argtypes = [C.c_void_p]
    L.cumc_slab_step_begin.argtypes = [C.c_void_p, C.c_double]
    L.cumc_slab_stage.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.cumc_slab_step_end.argtypes = [C.c_void_p]
    L.cumc_collapsar_get.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.cumc_learn_flags.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.cumc_learn_harvest.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p]
    L.cumc_mlp_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_void_p, C.c_void_p]
    L.cumc_mlp_train.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(capi.CumcTrainConfig), C.c_void_p, C.c_void_p]
    L.cumc_mlp_infer.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p]
    L.cumc_mlp_last_error.restype = C.c_char_p
    L.cumc_batch_run1_noalloc.argtypes = [C.POINTER(capi.CumcBatchConfig), C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_char_p, C.c_size_t]
    if path is None:
        _lib = L
    return L


class Solver:
    """One simulation on one GPU (a ``cumc_handle``)."""

    def __init__(self, spec):
        self.spec = spec
        self._cfg, self._keep = capi.make_config(spec)
        self.L = load_library()
        h = C.c_void_p()
        rc = self.L.cumc_create(C.byref(self._cfg), C.byref(h))
        if rc != 0:
            raise CumcError(rc, self.L.cumc_last_error(None).decode())
        self.h = h
        self.shape = (spec["nz"] + 6, spec["ny"] + 6, spec["nx"] + 6)
        self.time = 0.0
        self.n_step = 0

    def _check(self, rc):
        if rc != 0:
            raise CumcError(rc, self.L.cumc_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.cumc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # GET_MODEL output -> device
    def set_state(self, prim, eps):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        if prim.shape != self.shape + (8,) or eps.shape != self.shape:
            raise ValueError("state must have shape %s / %s" % (self.shape + (8,), self.shape))
        self._check(self.L.cumc_set_state(self.h, prim.ctypes.data, eps.ctypes.data))

    def get_state(self):
        prim = np.empty(self.shape + (8,))
        eps = np.empty(self.shape)
        self._check(self.L.cumc_get_state(self.h, prim.ctypes.data, eps.ctypes.data))
        return prim, eps

    def get_array(self, which):
        nc = {capi.ARR_CONS: 8, capi.ARR_BCELL: 3, capi.ARR_CS: 1}[which]
        out = np.empty(self.shape + ((nc,) if nc > 1 else ()))
        self._check(self.L.cumc_get_array(self.h, which, out.ctypes.data, out.size))
        return out

    def initial_update(self):
        self._check(self.L.cumc_initial_update(self.h))

    def finddt(self):
        dt = C.c_double()
        self._check(self.L.cumc_finddt(self.h, C.byref(dt)))
        return dt.value

    def rungekutta(self, dt):
        self._check(self.L.cumc_rk3_step(self.h, dt))

    def evolve(self, t_end, max_steps=2 ** 31 - 1):
        """main.f90:98-139 on the device; returns (time, steps taken)."""
        t = C.c_double(self.time)
        n = C.c_int(0)
        self._check(self.L.cumc_evolve(self.h, t_end, int(max_steps), C.byref(t), C.byref(n)))
        self.time = t.value
        self.n_step += n.value
        return t.value, n.value

    def find_divb(self):
        v = C.c_double()
        self._check(self.L.cumc_max_divb(self.h, C.byref(v)))
        return v.value

    def sync(self):
        self._check(self.L.cumc_sync(self.h))

    def launch_count(self):
        return int(self.L.cumc_launch_count(self.h))

    def stream(self):
        """The engine's cudaStream_t as an integer handle."""
        return int(self.L.cumc_stream(self.h) or 0)

    def profile_step(self, nsteps=1):
        """Per-kernel-class milliseconds summed over nsteps eager steps."""
        out = (C.c_double * 8)()
        self._check(self.L.cumc_profile_step(self.h, int(nsteps), out, 8))
        return dict(zip(PROFILE_CLASSES, list(out)))

    def autotune(self):
        """Pick the fastest face-flux launch shape on the live state."""
        ch = (C.c_int * 5)()
        ms = C.c_double()
        self._check(self.L.cumc_autotune(self.h, ch, C.byref(ms)))
        return dict(split=bool(ch[0]), tpb_recon=ch[1], tpb_riemann=ch[2], riemann_min_blocks=ch[3],
                    recon_tile=ch[4], flux_ms_per_stage=ms.value)

    def set_tuning(self, split=True, tpb_recon=256, tpb_riemann=128, riemann_min_blocks=1, recon_tile=0):
        ch = (C.c_int * 5)(int(split), tpb_recon, tpb_riemann, riemann_min_blocks, int(recon_tile))
        self._check(self.L.cumc_set_tuning(self.h, ch))

    def set_concurrent_sweeps(self, on=True):
        """Run each stage's three flux sweeps as concurrent branches (same bits)."""
        self._check(self.L.cumc_set_concurrent_sweeps(self.h, 1 if on else 0))

    def fallback_count(self, enable=-1):
        """Cells reconstructed with the positivity fallback since counting was
        enabled (enable=1 restarts from zero, 0 stops, -1 only reads)."""
        n = C.c_ulonglong()
        self._check(self.L.cumc_fallback_count(self.h, int(enable), C.byref(n)))
        return int(n.value)

    # ---- learned smooth-face flag (FP32 WENO form, handle created with learned=1) ----
    def learn_set(self, params, threshold=0.0, audit_interval=10, audit_tol=1e-6, flag_interval=1):
        """Enable the flag with these parameters (float[2657]); None disables it.
        The network runs every flag_interval steps; audits every audit_interval."""
        ptr = None
        if params is not None:
            P = np.ascontiguousarray(params, dtype=np.float32)
            if P.shape != (capi.LEARN_NP,):
                raise ValueError("parameters must have %d entries" % capi.LEARN_NP)
            ptr = P.ctypes.data
        self._check(self.L.cumc_learn_set(self.h, ptr, float(threshold), int(flag_interval), int(audit_interval),
                                          float(audit_tol)))

    def learn_stats(self):
        """Audit counters: cells audited, flagged, tiles set to fall back, audits."""
        out = (C.c_ulonglong * 4)()
        self._check(self.L.cumc_learn_stats(self.h, out))
        return dict(audited=out[0], flagged=out[1], fallback_tiles=out[2], audits=out[3])

    # ---- self-gravity potential of the collapsar model (spherical grids) ----
    def poisson_setup(self, rho_atm, omega=1.9):
        """Coefficients of the red-black SOR solver; phi = 0 everywhere."""
        self._check(self.L.cumc_poisson_setup(self.h, float(rho_atm), float(omega)))

    def poisson_solve(self, max_iter=100000, tol=1e-10):
        """Relax phi with the current density.  Returns (iterations, last
        max |dphi/phi_old|, converged)."""
        it, err, conv = C.c_int(), C.c_double(), C.c_int()
        self._check(self.L.cumc_poisson_solve(self.h, int(max_iter), float(tol), C.byref(it), C.byref(err),
                                              C.byref(conv)))
        return it.value, err.value, bool(conv.value)

    def poisson_get(self):
        """phi as (nz+2, ny+2, nx+2), cells 0..n+1 of each axis."""
        sp = self.spec
        out = np.empty((sp["nz"] + 2, sp["ny"] + 2, sp["nx"] + 2))
        self._check(self.L.cumc_poisson_get(self.h, out.ctypes.data))
        return out

    def poisson_set(self, phi):
        sp = self.spec
        P = np.ascontiguousarray(phi, dtype=np.float64)
        if P.shape != (sp["nz"] + 2, sp["ny"] + 2, sp["nx"] + 2):
            raise ValueError("phi must be (nz+2, ny+2, nx+2)")
        self._check(self.L.cumc_poisson_set(self.h, P.ctypes.data))

    # ---- output snapshots (print_hydroprofile's datasets, cumc_snapshot_*) ----
    def snapshot_start(self, primitive, epsilon, bfield):
        """Start copying the state into three float64 arrays (shapes of
        cumc3d_b200.snapshot.buffers; page-locked ones make it asynchronous).
        Keep them alive and untouched until snapshot_wait."""
        sp = self.spec
        shp = ((sp["nz"] + 2, sp["ny"] + 2, sp["nx"] + 2, 5), (sp["nz"] + 2, sp["ny"] + 2, sp["nx"] + 2),
               (sp["nz"] + 3, sp["ny"] + 3, sp["nx"] + 3, 3))
        for a, s in zip((primitive, epsilon, bfield), shp):
            if a.shape != s or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("snapshot buffer must be a contiguous float64 array of shape %s" % (s,))
        self._snap = (primitive, epsilon, bfield)  # kept alive while the copy runs
        self._check(self.L.cumc_snapshot_start(self.h, primitive.ctypes.data, epsilon.ctypes.data,
                                               bfield.ctypes.data))

    def snapshot_wait(self):
        self._check(self.L.cumc_snapshot_wait(self.h))
        self._snap = None

    def collapsar_set(self, m_bh, c_code):
        """The collapsar model's black hole: mass and c in code units."""
        self._check(self.L.cumc_collapsar_set(self.h, float(m_bh), float(c_code)))

    def collapsar_get(self):
        """(m_bh, r_sh) as the last stage left them."""
        m, r = C.c_double(), C.c_double()
        self._check(self.L.cumc_collapsar_get(self.h, C.byref(m), C.byref(r)))
        return m.value, r.value

    def learn_flags(self, direction):
        """The stored learned-flag state of one sweep: per-cell flags, per-warp
        linear decisions of the staged reconstruction, per-tile fallback marks."""
        sizes = (C.c_longlong * 3)()
        self._check(self.L.cumc_learn_flags(self.h, int(direction), None, None, None, sizes))
        f, w, t = (np.empty(int(n), dtype=np.uint8) for n in sizes)
        self._check(self.L.cumc_learn_flags(self.h, int(direction), f.ctypes.data, w.ctypes.data, t.ctypes.data,
                                            sizes))
        return f, w, t

    def learn_harvest(self, direction, stride=1):
        """Samples (rows of 37 floats) of every stride-th interior cell, one sweep."""
        n = self.spec["nx"] * self.spec["ny"] * self.spec["nz"]
        rows = (n + stride - 1) // stride
        out = np.empty((rows, capi.LEARN_ROW), dtype=np.float32)
        got = C.c_longlong()
        self._check(self.L.cumc_learn_harvest(self.h, int(direction), int(stride), out.ctypes.data, rows,
                                              C.byref(got)))
        return out[:got.value]

    def set_state_ptr(self, prim_ptr, eps_ptr):
        """set_state from raw host pointers (e.g. pinned buffers)."""
        self._check(self.L.cumc_set_state(self.h, prim_ptr, eps_ptr))

    def get_state_ptr(self, prim_ptr, eps_ptr):
        self._check(self.L.cumc_get_state(self.h, prim_ptr, eps_ptr))


class BatchSolver:
    """Many independent 1D problems (each a reference n_dim = 1 run of
    solver/mhd/main.f90) advanced in one persistent launch.

    ``specs`` are 1D specs (ny = nz = 1, outflow everywhere, Cartesian) that
    share cfl, gamma, the scheme and the precision; each keeps its own grid,
    initial state and ``t_end``.
    """

    def __init__(self, specs, positivity_fallback=0):
        if not specs:
            raise ValueError("no problems")
        s0 = specs[0]
        for sp in specs:
            if sp["ny"] != 1 or sp["nz"] != 1 or sp["n_dim"] != 1 or sp.get("coordinate_flag", 0) != 0:
                raise ValueError("batched problems are 1D Cartesian")
            if tuple(sp["boundary_flag"]) != (1, 1, 1, 1, 1, 1):
                raise ValueError("batched problems use outflow boundaries")
            for key in ("cfl", "recon", "riemann", "precision"):
                if sp[key] != s0[key]:
                    raise ValueError("batched problems must share %s" % key)
            if sp["model"].get("gamma") != s0["model"].get("gamma"):
                raise ValueError("batched problems must share gamma")
        self.L = load_library()
        self.specs = specs
        self.n = [int(sp["nx"]) for sp in specs]
        self._xf = [np.ascontiguousarray(sp["xF"], dtype=np.float64) for sp in specs]
        nprob = len(specs)
        self._nx = (C.c_int * nprob)(*self.n)
        self._xfp = (C.POINTER(C.c_double) * nprob)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in self._xf])
        self._tend = (C.c_double * nprob)(*[float(sp["t_end"]) for sp in specs])
        cfg = capi.CumcBatchConfig()
        cfg.n_problems = nprob
        cfg.nx = self._nx
        cfg.xF = self._xfp
        cfg.t_end = self._tend
        cfg.cfl = float(s0["cfl"])
        cfg.gamma = float(s0["model"].get("gamma", 5.0 / 3.0))
        cfg.recon = capi.RECON[s0["recon"]]
        cfg.riemann = capi.RIEMANN[s0["riemann"]]
        cfg.precision = capi.PRECISION[s0["precision"]]
        cfg.floor_kind = capi.FLOOR[s0["model"].get("floor", "eps")]
        cfg.positivity_fallback = int(positivity_fallback)
        self._cfg = cfg
        h = C.c_void_p()
        rc = self.L.cumc_batch_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise CumcError(rc, self.L.cumc_batch_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise CumcError(rc, self.L.cumc_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.cumc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, p, prim, eps):
        """GET_MODEL output of problem p, shape (7, 7, n+6, 8) / (7, 7, n+6)."""
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        shape = (7, 7, self.n[p] + 6)
        if prim.shape != shape + (8,) or eps.shape != shape:
            raise ValueError("state of problem %d must have shape %s" % (p, shape))
        self._check(self.L.cumc_batch_set_state(self.h, p, prim.ctypes.data, eps.ctypes.data))

    def get_state(self, p):
        """(prim (n+6, 8), eps (n+6,)) of the (k, l) = (1, 1) row of problem p."""
        prim = np.empty((self.n[p] + 6, 8))
        eps = np.empty(self.n[p] + 6)
        self._check(self.L.cumc_batch_get_state(self.h, p, prim.ctypes.data, eps.ctypes.data))
        return prim, eps

    def run(self, max_steps=0, check=True):
        """INITIAL_UPDATE + every time loop; returns (t, steps, status) arrays.

        A problem that reaches a non-finite or non-positive state stops there
        with status CUMC_ESTATE; with ``check`` the call then raises, without
        it the per-problem results are returned as they are."""
        m = len(self.n)
        t = np.zeros(m)
        steps = np.zeros(m, dtype=np.int32)
        status = np.zeros(m, dtype=np.int32)
        rc = self.L.cumc_batch_run(self.h, int(max_steps), t.ctypes.data, steps.ctypes.data, status.ctypes.data)
        if rc != 0 and (check or rc != capi.CUMC_ESTATE):
            self._check(rc)
        return t, steps, status

    def set_cluster(self, cluster_size=8, coop_min_n=1024):
        """CTAs per cluster for problems of more than coop_min_n cells
        (smaller ones run one per CTA); results do not depend on it."""
        self._check(self.L.cumc_batch_set_cluster(self.h, int(cluster_size), int(coop_min_n)))

    def sync(self):
        self._check(self.L.cumc_batch_sync(self.h))

    def stream(self):
        return int(self.L.cumc_batch_stream(self.h) or 0)

    def launch_count(self):
        """Kernel launches issued since creation."""
        return int(self.L.cumc_batch_launch_count(self.h))


def batch_run1_noalloc(spec, prim, eps, max_steps=0, positivity_fallback=0, stream=0):
    """One 1D problem through ``cumc_batch_run1_noalloc`` (no device
    allocation; at most 4096 zones).  Returns (prim row (n+6, 8), eps row,
    t, steps); raises CumcError on a non-zero status."""
    L = load_library()
    n = int(spec["nx"])
    xf = np.ascontiguousarray(spec["xF"], dtype=np.float64)
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    if prim.shape != (7, 7, n + 6, 8) or eps.shape != (7, 7, n + 6):
        raise ValueError("state must have shape (7, 7, n+6, 8) / (7, 7, n+6)")
    nx = (C.c_int * 1)(n)
    xfp = (C.POINTER(C.c_double) * 1)(xf.ctypes.data_as(C.POINTER(C.c_double)))
    tend = (C.c_double * 1)(float(spec["t_end"]))
    cfg = capi.CumcBatchConfig()
    cfg.n_problems = 1
    cfg.nx = nx
    cfg.xF = xfp
    cfg.t_end = tend
    cfg.cfl = float(spec["cfl"])
    cfg.gamma = float(spec["model"].get("gamma", 5.0 / 3.0))
    cfg.recon = capi.RECON[spec["recon"]]
    cfg.riemann = capi.RIEMANN[spec["riemann"]]
    cfg.precision = capi.PRECISION[spec["precision"]]
    cfg.floor_kind = capi.FLOOR[spec["model"].get("floor", "eps")]
    cfg.positivity_fallback = int(positivity_fallback)
    prow = np.empty((n + 6, 8))
    erow = np.empty(n + 6)
    t = C.c_double()
    steps = C.c_int()
    status = C.c_int()
    err = C.create_string_buffer(256)
    rc = L.cumc_batch_run1_noalloc(C.byref(cfg), prim.ctypes.data, eps.ctypes.data, int(max_steps),
                                   C.c_void_p(stream), prow.ctypes.data, erow.ctypes.data, C.addressof(t),
                                   C.addressof(steps), C.addressof(status), err, 256)
    if rc != 0:
        raise CumcError(rc, err.value.decode())
    return prow, erow, t.value, steps.value


def _mlp_check(L, rc):
    if rc != 0:
        raise CumcError(rc, L.cumc_mlp_last_error().decode())


def mlp_init(seed=0):
    """He-uniform initial parameters of the flag network (inputs 35..47 zero)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(capi.LEARN_NP, dtype=np.float32)
    lim1 = np.sqrt(6.0 / capi.LEARN_NF)
    W1 = np.zeros((32, 48), dtype=np.float32)
    W1[:, :capi.LEARN_NF] = rng.uniform(-lim1, lim1, (32, capi.LEARN_NF))
    P[0:1536] = W1.ravel()
    lim2 = np.sqrt(6.0 / 32)
    P[1568:2592] = rng.uniform(-lim2, lim2, 32 * 32)
    P[2624:2656] = rng.uniform(-lim2, lim2, 32)
    return P


def mlp_grad(params, samples, delta):
    """(mean loss, gradient) of the flag network on the GPU (FP32)."""
    L = load_library()
    P = np.ascontiguousarray(params, dtype=np.float32)
    S = np.ascontiguousarray(samples, dtype=np.float32)
    g = np.zeros(capi.LEARN_NP, dtype=np.float32)
    loss = C.c_float()
    _mlp_check(L, L.cumc_mlp_grad(P.ctypes.data, S.ctypes.data, S.shape[0], float(delta), g.ctypes.data,
                                  C.byref(loss)))
    return loss.value, g


def mlp_train(samples, params, steps=2000, batch=4096, lr=1e-3, delta=1e-6, seed=1):
    """Adam on the GPU; returns (parameters, loss per step)."""
    L = load_library()
    P = np.array(params, dtype=np.float32, copy=True)
    S = np.ascontiguousarray(samples, dtype=np.float32)
    tc = capi.CumcTrainConfig(steps=int(steps), batch=int(batch), lr=float(lr), delta=float(delta), beta1=0.0,
                              beta2=0.0, eps=0.0, seed=int(seed))
    losses = np.zeros(int(steps), dtype=np.float32)
    _mlp_check(L, L.cumc_mlp_train(S.ctypes.data, S.shape[0], C.byref(tc), P.ctypes.data, losses.ctypes.data))
    return P, losses


def mlp_infer(params, features):
    """Logits of feature rows on the tensor cores (the reconstruction kernel's MLP)."""
    L = load_library()
    P = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(features, dtype=np.float32)
    z = np.zeros(X.shape[0], dtype=np.float32)
    _mlp_check(L, L.cumc_mlp_infer(P.ctypes.data, X.ctypes.data, X.shape[1], X.shape[0], z.ctypes.data))
    return z


def fp64_peak_tflops():
    v = C.c_double()
    rc = load_library().cumc_fp64_peak(C.byref(v))
    if rc != 0:
        raise CumcError(rc, "fp64 peak probe failed")
    return v.value


def check_div3(seed, n):
    """(mismatches, example input) of the FMA-corrected x/3 against IEEE x/3."""
    m = C.c_ulonglong()
    ex = C.c_double()
    rc = load_library().cumc_check_div3(seed, n, C.byref(m), C.byref(ex))
    if rc != 0:
        raise CumcError(rc, "div3 check failed to run")
    return m.value, ex.value


def slab_specs(spec, sizes):
    """The per-slab specs of a z cut: each slab's z faces are its cells plus
    three ghost faces per side, a sub-array of the whole grid's zF; a side
    shared with a neighbour is marked BOUNDARY_EXCHANGE (both ends too when
    z is periodic: the slabs form a ring).  Returns (specs, z offsets)."""
    if sum(sizes) != spec["nz"] or min(sizes) < 3:
        raise ValueError("slab sizes must be >= 3 and sum to nz")
    bf = list(spec["boundary_flag"])
    ring = bf[4] == 0
    offsets = [sum(sizes[:i]) for i in range(len(sizes))]
    out = []
    for i, (o, m) in enumerate(zip(offsets, sizes)):
        sp = dict(spec)
        sp["nz"] = m
        sp["zF"] = np.asarray(spec["zF"])[o:o + m + 7]   # faces -3..m+3 of the slab
        f = list(bf)
        f[4] = capi.BOUNDARY_EXCHANGE if (i > 0 or ring) else bf[4]
        f[5] = capi.BOUNDARY_EXCHANGE if (i + 1 < len(sizes) or ring) else bf[5]
        sp["boundary_flag"] = f
        out.append(sp)
    return out, offsets


class SlabGroup:
    """One grid cut along z into slabs, one Solver per slab (cumc_group_*).

    sizes: the slabs' z cell counts (summing to spec["nz"]); devices: a CUDA
    device per slab (None: the current one).  A periodic z axis makes the
    slabs a ring.  set_state / get_state take and give the whole grid's
    arrays (prim (nz+6, ny+6, nx+6, 8), eps (nz+6, ny+6, nx+6)); the group's
    state equals the undivided grid's bit for bit."""

    def __init__(self, spec, sizes, devices=None):
        specs, self.offsets = slab_specs(spec, sizes)
        self.spec, self.sizes = spec, list(sizes)
        self.devices = list(devices) if devices is not None else None
        self.slabs = []
        for i, sp in enumerate(specs):
            with self._on(i):
                self.slabs.append(Solver(sp))
        self.L = self.slabs[0].L
        self._arr = (C.c_void_p * len(self.slabs))(*[s.h for s in self.slabs])

    def _on(self, i):
        """Context with slab i's GPU current (calls on a handle run on its GPU)."""
        import contextlib
        if self.devices is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.device(self.devices[i])

    def _check(self, rc):
        if rc != 0:
            raise CumcError(rc, self.L.cumc_last_error(self.slabs[0].h).decode())

    def set_state(self, prim, eps):
        for i, (s, o, m) in enumerate(zip(self.slabs, self.offsets, self.sizes)):
            with self._on(i):
                s.set_state(np.ascontiguousarray(prim[o:o + m + 6]), np.ascontiguousarray(eps[o:o + m + 6]))

    def initial_update(self):
        self._check(self.L.cumc_group_initial_update(self._arr, len(self.slabs)))

    def finddt(self):
        dt = C.c_double()
        self._check(self.L.cumc_group_finddt(self._arr, len(self.slabs), C.byref(dt)))
        return dt.value

    def step(self, dt):
        self._check(self.L.cumc_group_step(self._arr, len(self.slabs), float(dt)))

    def _gather(self, parts):
        """Interior planes of every slab, in z order (axis 0 of the padded
        arrays), as the whole grid's interior."""
        return np.concatenate([p[3:3 + m] for p, m in zip(parts, self.sizes)], axis=0)

    def get_state(self):
        """(prim, eps) of the interior cells, (nz, ny+6, nx+6, ...)."""
        st = []
        for i, s in enumerate(self.slabs):
            with self._on(i):
                st.append(s.get_state())
        return self._gather([p for p, _ in st]), self._gather([e for _, e in st])

    def get_array(self, which):
        parts = []
        for i, s in enumerate(self.slabs):
            with self._on(i):
                parts.append(s.get_array(which))
        return self._gather(parts)

    def close(self):
        for i, s in enumerate(self.slabs):
            with self._on(i):
                s.close()


FILL_STATE, FILL_EMF = 0, 1  # the two exchange points of a stage (CUMC_FILL_*)


def halo_peers(rank, n, ring):
    """(lower, upper) neighbour ranks of slab `rank` of n along z; None on a
    side that is a boundary of the whole grid."""
    lo = rank - 1 if rank > 0 else (n - 1 if ring else None)
    hi = rank + 1 if rank + 1 < n else (0 if ring else None)
    return lo, hi


def halo_p2p_ops(peers, send, recv, group=None, tags=True):
    """torch.distributed point-to-point ops of one exchange point.  send /
    recv: side -> buffer.  What a rank packs at side s its neighbour unpacks
    at side 1 - s.  Sends are posted in side order 0, 1 and receives in side
    order 1, 0: in a ring of two slabs both neighbours are the same rank and
    the two messages between a pair are matched in posting order (NCCL), so
    this order pairs the lower planes with the upper ghosts; the tags (the
    sender's side) pair them the same way where tags are honoured (gloo;
    tags=False leaves matching to the posting order alone)."""
    import torch.distributed as dist
    ops = [dist.P2POp(dist.isend, send[s], peers[s], group, tag=s if tags else 0)
           for s in (0, 1) if peers[s] is not None]
    ops += [dist.P2POp(dist.irecv, recv[s], peers[s], group, tag=(1 - s) if tags else 0)
            for s in (1, 0) if peers[s] is not None]
    return ops


class SlabRank:
    """One slab of a z-cut grid per process: the one-rank-per-GPU form of
    SlabGroup (cumc_slab_*).  spec / sizes as for SlabGroup (the whole grid,
    the slabs' z cell counts); this process holds slab `rank`, on the current
    CUDA device.  The ghost planes travel by torch.distributed send/recv of
    contiguous device buffers (NCCL over NVLink between GPUs), or through
    pinned host buffers when the process group's backend is not NCCL (gloo,
    e.g. several ranks on one GPU).  finddt is the minimum over the ranks
    (an all-reduce).  The ranks' states equal the undivided grid's bit for
    bit."""

    def __init__(self, spec, sizes, rank, group=None):
        import torch
        specs, offsets = slab_specs(spec, sizes)
        if len(sizes) < 2:
            raise ValueError("a z cut needs at least two slabs")
        self.n, self.rank, self.group = len(sizes), rank, group
        self.offset, self.size = offsets[rank], sizes[rank]
        ring = spec["boundary_flag"][4] == 0
        self.peers = halo_peers(rank, self.n, ring)
        self.solver = Solver(specs[rank])
        self.L, self.h = self.solver.L, self.solver.h
        if ring and rank == 0:
            self._check(self.L.cumc_slab_seam(self.h, 0))
        if ring and rank == self.n - 1:
            self._check(self.L.cumc_slab_seam(self.h, 1))
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._stream = torch.cuda.ExternalStream(self.solver.stream(), device=self.device)
        self.send, self.recv = {}, {}
        for fill in (FILL_STATE, FILL_EMF):
            for side in (0, 1):
                if self.peers[side] is None:
                    continue
                nb = C.c_size_t()
                self._check(self.L.cumc_slab_halo_bytes(self.h, fill, side, C.byref(nb)))
                self.send[fill, side] = torch.empty(nb.value, dtype=torch.uint8, device=self.device)
                self.recv[fill, side] = torch.empty(nb.value, dtype=torch.uint8, device=self.device)
        self._staged = None
        self.time, self.n_step = 0.0, 0

    def _check(self, rc):
        if rc != 0:
            raise CumcError(rc, self.L.cumc_last_error(self.h).decode())

    # -- the per-rank calls (one exchange point = pack, transport, unpack) --
    def pack(self, fill):
        for side in (0, 1):
            if self.peers[side] is not None:
                self._check(self.L.cumc_slab_halo_pack(self.h, fill, side, self.send[fill, side].data_ptr()))

    def unpack(self, fill):
        for side in (0, 1):
            if self.peers[side] is not None:
                self._check(self.L.cumc_slab_halo_unpack(self.h, fill, side, self.recv[fill, side].data_ptr()))

    def stage(self, stage, part):
        self._check(self.L.cumc_slab_stage(self.h, stage, part))

    def initial_begin(self):
        self._check(self.L.cumc_slab_initial_begin(self.h))

    def initial_end(self):
        self._check(self.L.cumc_slab_initial_end(self.h))

    def step_begin(self, dt):
        self._check(self.L.cumc_slab_step_begin(self.h, float(dt)))

    def step_end(self):
        self._check(self.L.cumc_slab_step_end(self.h))

    # -- torch.distributed driver --
    def _transport(self, fill):
        import torch
        import torch.distributed as dist
        if self._staged is None:
            self._staged = dist.get_backend(self.group) != "nccl"
            if self._staged:
                self._hsend = {k: torch.empty(v.numel(), dtype=torch.uint8, pin_memory=True) for k, v in self.send.items()}
                self._hrecv = {k: torch.empty(v.numel(), dtype=torch.uint8, pin_memory=True) for k, v in self.recv.items()}
        sides = [s for s in (0, 1) if self.peers[s] is not None]
        if not self._staged:
            # NCCL runs on its own stream, after the packs on the engine's
            # stream; wait() orders the engine's stream after it
            with torch.cuda.stream(self._stream):
                works = dist.batch_isend_irecv(halo_p2p_ops(self.peers, {s: self.send[fill, s] for s in sides},
                                                            {s: self.recv[fill, s] for s in sides}, self.group))
                for w in works:
                    w.wait()
            return
        with torch.cuda.stream(self._stream):
            for s in sides:
                self._hsend[fill, s].copy_(self.send[fill, s], non_blocking=True)
        self._stream.synchronize()
        works = dist.batch_isend_irecv(halo_p2p_ops(self.peers, {s: self._hsend[fill, s] for s in sides},
                                                    {s: self._hrecv[fill, s] for s in sides}, self.group))
        for w in works:
            w.wait()
        with torch.cuda.stream(self._stream):
            for s in sides:
                self.recv[fill, s].copy_(self._hrecv[fill, s], non_blocking=True)

    def exchange(self, fill):
        self.pack(fill)
        self._transport(fill)
        self.unpack(fill)

    def set_state(self, prim, eps):
        """The whole grid's prim (nz+6, ny+6, nx+6, 8) and eps; this rank
        takes its planes."""
        o, m = self.offset, self.size
        self.solver.set_state(np.ascontiguousarray(prim[o:o + m + 6]), np.ascontiguousarray(eps[o:o + m + 6]))

    def initial_update(self):
        self.initial_begin()
        self.exchange(FILL_STATE)
        self.initial_end()

    def finddt(self):
        import torch
        import torch.distributed as dist
        dt = self.solver.finddt()
        t = torch.tensor([dt], dtype=torch.float64, device="cpu" if self._is_staged() else self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())

    def _is_staged(self):
        if self._staged is None:
            import torch.distributed as dist
            return dist.get_backend(self.group) != "nccl"
        return self._staged

    def step(self, dt):
        self.step_begin(dt)
        for stage in (1, 2, 3):
            self.stage(stage, 0)
            self.exchange(FILL_EMF)
            self.stage(stage, 1)
            self.exchange(FILL_STATE)
        self.step_end()
        self.time += dt
        self.n_step += 1

    def get_state(self):
        """(prim, eps) of this slab's interior planes, (size, ny+6, nx+6, ...)."""
        p, e = self.solver.get_state()
        return p[3:3 + self.size], e[3:3 + self.size]

    def get_array(self, which):
        return self.solver.get_array(which)[3:3 + self.size]

    def close(self):
        """Release the halo buffers while the engine's stream still exists
        (freeing a buffer that a copy used records an event on that stream),
        then the handle."""
        import torch
        self._stream.synchronize()
        self.send, self.recv = {}, {}
        self._hsend, self._hrecv = {}, {}
        torch.cuda.synchronize(self.device)
        self.solver.close()


def check_dv(seed, n):
    """(mismatches, (x, y) of one differing pair) of the engine's FP64
    division against the IEEE quotient x / y."""
    m = C.c_ulonglong()
    ex = (C.c_double * 2)()
    rc = load_library().cumc_check_dv(seed, n, C.byref(m), ex)
    if rc != 0:
        raise CumcError(rc, "dv check failed to run")
    return m.value, (ex[0], ex[1])
