"""ctypes front end of the CPU oracle (oracle/cumc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product package.

PARITY UNPINNED: the reference is Fortran and cannot be built here (no
Fortran compiler); it ships no golden vectors.  The oracle is a line-by-line
restatement checked by invariants (tests/test_oracle_invariants.py) and by
known answers (the exact Riemann solution on the Toro tubes,
tests/test_riemann1d.py; the CP Alfven wave after one period).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
SRC = os.path.join(HERE, "cumc_oracle.cpp")

# parity recipe: no FP contraction (bitwise order is kept), OpenMP loops as in
# the reference's CPU build, generic x86-64 code (the library travels).
CXXFLAGS = ["-std=c++17", "-O3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared"]
# timed recipe of the CPU baseline: the same plus -march=native, compiled on
# the host that runs it (the code it emits may not run on another CPU); the
# arithmetic is the same (no contraction, no fast-math), only vectorised
NATIVE_DIR = os.path.join(BUILD, "native")
NATIVE_LIB = os.path.join(NATIVE_DIR, "liboracle.so")


def _deps_mtime():
    return max(os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "..", "include", "cumc3d_gpu.h")))


def build(force=False):
    os.makedirs(BUILD, exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _deps_mtime():
        subprocess.check_call(["g++"] + CXXFLAGS + ["-o", LIB, SRC])
    return LIB


def _cpu_key():
    """Model name and flags of this host's CPU (the native build's target)."""
    try:
        with open("/proc/cpuinfo") as f:
            txt = f.read()
    except OSError:
        return "unknown"
    keep = [ln for ln in txt.splitlines() if ln.startswith(("model name", "flags"))][:2]
    return "\n".join(keep)


def use_native():
    """Switch this process to the -march=native build (compiled here on first
    use, again when the host CPU differs from the one it was built for).
    Must be called before the first Oracle is made.  Returns a description of
    the recipe in use; on a compiler failure the generic build stays."""
    global LIB
    if _lib is not None:
        return "generic (-O3, the library was already loaded)"
    os.makedirs(NATIVE_DIR, exist_ok=True)
    stamp = os.path.join(NATIVE_DIR, "cpu.txt")
    key = _cpu_key()
    old = open(stamp).read() if os.path.exists(stamp) else None
    if old != key or not os.path.exists(NATIVE_LIB) or os.path.getmtime(NATIVE_LIB) < _deps_mtime():
        try:
            subprocess.check_call(["g++"] + CXXFLAGS + ["-march=native", "-o", NATIVE_LIB, SRC])
        except (OSError, subprocess.CalledProcessError) as ex:
            return "generic (-O3; the -march=native build failed: %s)" % ex
        with open(stamp, "w") as f:
            f.write(key)
    LIB = NATIVE_LIB
    return "g++ -O3 -march=native -ffp-contract=off -fno-fast-math -fopenmp"


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_fallback_count.argtypes = [C.c_void_p]
        L.orc_fallback_count.restype = C.c_ulonglong
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.c_int]
        L.orc_last_error.restype = C.c_char_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_get_array.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_initial_update.argtypes = [C.c_void_p]
        L.orc_finddt.argtypes = [C.c_void_p]
        L.orc_finddt.restype = C.c_double
        L.orc_rk3_step.argtypes = [C.c_void_p, C.c_double]
        L.orc_evolve.argtypes = [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.orc_evolve.restype = C.c_int
        L.orc_max_divb.argtypes = [C.c_void_p]
        L.orc_max_divb.restype = C.c_double
        L.orc_get_counts.argtypes = [C.POINTER(C.c_uint64)]
        L.orc_get_phase_counts.argtypes = [C.c_int, C.POINTER(C.c_uint64)]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        L.orc_recon_cell.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_weights.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.orc_riemann_face.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_learn_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p]
        L.orc_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_void_p]
        L.orc_mlp_loss_grad.restype = C.c_double
        L.orc_poisson_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_poisson_solve.restype = C.c_int
        L.orc_collapsar_set.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.orc_collapsar_get.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_collapsar_get.restype = C.c_int
        L.orc_set_phi.argtypes = [C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """Mirror of the engine's host API, running the CPU restatement."""

    def __init__(self, spec, counting=False):
        from cumc3d_b200.capi import make_config  # structures only
        self.spec = spec
        self._cfg, self._keep = make_config(spec)
        L = lib()
        self.h = L.orc_create(C.byref(self._cfg), 1 if counting else 0)
        if not self.h:
            raise ValueError("oracle create failed: %s" % L.orc_last_error().decode())
        self.shape = (spec["nz"] + 6, spec["ny"] + 6, spec["nx"] + 6)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, prim, eps):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        assert prim.shape == self.shape + (8,) and eps.shape == self.shape
        lib().orc_set_state(self.h, prim.ctypes.data, eps.ctypes.data)

    def fallback_count(self):
        """Cells reconstructed with the positivity fallback so far."""
        return int(lib().orc_fallback_count(self.h))

    def get_state(self):
        prim = np.empty(self.shape + (8,))
        eps = np.empty(self.shape)
        lib().orc_get_state(self.h, prim.ctypes.data, eps.ctypes.data)
        return prim, eps

    def get_array(self, which):
        ncomp = {0: 8, 1: 3, 2: 1}[which]
        out = np.empty(self.shape + ((ncomp,) if ncomp > 1 else ()))
        lib().orc_get_array(self.h, which, out.ctypes.data)
        return out

    def initial_update(self):
        lib().orc_initial_update(self.h)

    def finddt(self):
        return lib().orc_finddt(self.h)

    def rk3_step(self, dt):
        lib().orc_rk3_step(self.h, dt)

    def evolve(self, t_end, max_steps, t=0.0):
        tt = C.c_double(t)
        n = lib().orc_evolve(self.h, t_end, max_steps, C.byref(tt))
        return tt.value, n

    def collapsar_set(self, m_bh, c_code):
        lib().orc_collapsar_set(self.h, float(m_bh), float(c_code))

    def collapsar_get(self):
        """(m_bh, r_sh, horizon reached the inner face)."""
        m, r = C.c_double(), C.c_double()
        hit = lib().orc_collapsar_get(self.h, C.byref(m), C.byref(r))
        return m.value, r.value, bool(hit)

    def set_phi(self, phi):
        sp = self.spec
        P = np.ascontiguousarray(phi, dtype=np.float64)
        assert P.shape == (sp["nz"] + 2, sp["ny"] + 2, sp["nx"] + 2)
        lib().orc_set_phi(self.h, P.ctypes.data)

    def max_divb(self):
        return lib().orc_max_divb(self.h)


def reset_counts():
    lib().orc_reset_counts()


PHASES = {"other": 0, "recon": 1, "riemann": 2, "finddt": 3}


def get_counts(phase=None):
    """Operations of a counting handle since reset_counts: all phases, or
    one of PHASES ("recon": face reconstruction; "riemann": BUILDSTATES and
    the Riemann solver; "finddt"; "other": the rest of the step)."""
    out = (C.c_uint64 * 5)()
    lib().orc_get_phase_counts(-1 if phase is None else PHASES[phase], out)
    return dict(add=out[0], mul=out[1], div=out[2], sqrt=out[3], cmp=out[4])


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def weights(rec, d5):
    d5 = np.ascontiguousarray(d5, dtype=np.float64)
    w = np.zeros(14)
    lib().orc_weights(rec, d5.ctypes.data, w.ctypes.data)
    return w


def recon_cell(rec, w, v5):
    w = np.ascontiguousarray(w, dtype=np.float64)
    v5 = np.ascontiguousarray(v5, dtype=np.float64)
    vm, vp = C.c_double(), C.c_double()
    lib().orc_recon_cell(rec, w.ctypes.data, v5.ctypes.data, C.byref(vm), C.byref(vp))
    return vm.value, vp.value


def riemann_face(dir_, rs, gamma, pl, pr):
    """(Riemann flux, physical flux of the left state) for one face; dir_ 1..3."""
    pl = np.ascontiguousarray(pl, dtype=np.float64)
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    fo = np.zeros(8)
    fp = np.zeros(8)
    lib().orc_riemann_face(dir_, rs, gamma, pl.ctypes.data, pr.ctypes.data, fo.ctypes.data, fp.ctypes.data)
    return fo, fp


# ---------------------------------------------------------------------------
# learned smooth-face flag: the checker of the GPU harvest, trainer, inference
# ---------------------------------------------------------------------------
LEARN_NP, LEARN_NF, LEARN_ROW = 2657, 35, 37


def learn_sample(stencils, w10):
    """stencils (7, 5) FP64, w10 the cell's WENO weights -> 37-float sample row."""
    st = np.ascontiguousarray(stencils, dtype=np.float64)
    w = np.ascontiguousarray(w10, dtype=np.float64)
    row = np.zeros(LEARN_ROW, dtype=np.float32)
    lib().orc_learn_sample(st.ctypes.data, w.ctypes.data, row.ctypes.data)
    return row


def mlp_forward(params, X):
    """FP64 forward pass of the flag network on rows of features."""
    P = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    z = np.zeros(X.shape[0])
    lib().orc_mlp_forward(P.ctypes.data, X.ctypes.data, X.shape[1], X.shape[0], z.ctypes.data)
    return z


def mlp_loss_grad(params, samples, delta):
    """FP64 mean binary cross-entropy of "change < delta" and its gradient."""
    P = np.ascontiguousarray(params, dtype=np.float32)
    S = np.ascontiguousarray(samples, dtype=np.float32)
    assert S.shape[1] == LEARN_ROW
    g = np.zeros(LEARN_NP)
    loss = lib().orc_mlp_loss_grad(P.ctypes.data, S.ctypes.data, S.shape[0], delta, g.ctypes.data)
    return loss, g


def _bf16(a):
    """Round FP32 values to BF16 (nearest even), returned as FP32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def mlp_forward_bf16(params, X):
    """The tensor-core inference emulated: BF16 features, W1, hidden layer and
    W2, FP32 accumulation (in FP64 here), FP32 output layer."""
    P = np.asarray(params, dtype=np.float32)
    W1 = _bf16(P[0:1536]).reshape(32, 48).astype(np.float64)
    b1 = P[1536:1568].astype(np.float64)
    W2 = _bf16(P[1568:2592]).reshape(32, 32).astype(np.float64)
    b2 = P[2592:2624].astype(np.float64)
    w3 = P[2624:2656].astype(np.float64)
    b3 = float(P[2656])
    x = np.zeros((X.shape[0], 48), dtype=np.float32)
    x[:, :LEARN_NF] = X[:, :LEARN_NF]
    h1 = np.maximum(_bf16(x).astype(np.float64) @ W1.T + b1, 0.0)
    h1 = _bf16(h1.astype(np.float32)).astype(np.float64)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ w3 + b3


def poisson_solve(spec, rho, rho_atm, omega=1.9, tol=1e-10, max_iter=100000, phi=None):
    """Red-black SOR for the collapsar self-gravity potential (the oracle's
    restatement of model/collapsar/src/custom.f90:511-620).  rho: interior
    (nz, ny, nx); phi: (nz+2, ny+2, nx+2) start value (zeros if None).
    Returns (phi, iterations, last error, converged)."""
    from cumc3d_b200.capi import make_config  # structures only
    cfg, keep = make_config(spec)
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    r = np.ascontiguousarray(rho, dtype=np.float64).reshape(nz, ny, nx)
    p = np.zeros((nz + 2, ny + 2, nx + 2)) if phi is None else np.array(phi, dtype=np.float64, copy=True)
    it, err = C.c_int(), C.c_double()
    conv = lib().orc_poisson_solve(C.byref(cfg), r.ctypes.data, float(rho_atm), float(omega), float(tol),
                                   int(max_iter), p.ctypes.data, C.byref(it), C.byref(err))
    del keep
    return p, it.value, err.value, bool(conv)
