"""A compiled C host program on the GPU: cumc3d_b200/host/cumc_main.c builds
the Brio-Wu tube itself, links the engine library and replays the
reference's main loop (solver/mhd/main.f90:98-139: FINDDT, the clamp to
total_time, RUNGEKUTTA) through the C-ABI alone -- no Python between the
host and the engine.  Its final state must equal the CPU oracle's run of the
same model (built here by the Python model code) bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from cumc3d_b200 import engine, models
from parity_util import interior

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_host_replays_main_loop_bitwise(oracle_mod, tmp_path):
    engine.load_library()  # builds are in-tree; make sure the library exists
    exe = str(tmp_path / "cumc_main")
    lib = engine.LIB_PATH
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "cumc3d_b200", "host", "cumc_main.c"), lib,
                    "-Wl,-rpath," + os.path.dirname(lib), "-lm", "-o", exe], check=True)
    nx = 128
    out = str(tmp_path / "state.bin")
    r = subprocess.run([exe, str(nx), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    words = r.stdout.split()
    steps, t = int(words[1]), float(words[3])
    spec, prim, eps = models.brio_wu(nx)
    o = oracle_mod.Oracle(spec)
    o.set_state(prim, eps)
    o.initial_update()
    to, no = o.evolve(0.1, 10 ** 6)
    assert (steps, t) == (no, to) and t == 0.1
    raw = np.fromfile(out, dtype=np.float64)
    n3 = (nx + 6) * 7 * 7
    pg = raw[:8 * n3].reshape(7, 7, nx + 6, 8)
    eg = raw[8 * n3:].reshape(7, 7, nx + 6)
    po, eo = o.get_state()
    assert np.array_equal(interior(pg, spec), interior(po, spec))
    assert np.array_equal(interior(eg, spec), interior(eo, spec))
    o.close()
