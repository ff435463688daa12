"""C-ABI boundary checks that need no GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from cumc3d_b200 import capi, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cumc3d_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cumc_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = engine.LIB_PATH
    assert os.path.exists(lib), "build the engine first (python -m cumc3d_b200.build)"
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, "not exported: %s" % missing
    assert sorted(engine.EXPORTS) == declared_functions()


def test_library_loads_and_binds():
    L = engine.load_library()
    for name in engine.EXPORTS:
        assert hasattr(L, name)


def test_struct_layout_matches_header():
    # sizes of the C structs, compiled from the header with the host compiler
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "cumc3d_gpu.h"
int main(void){printf("%zu %zu %zu %zu %zu\n", sizeof(cumc_model), sizeof(cumc_config),
 offsetof(cumc_config, xF), offsetof(cumc_config, cfl), offsetof(cumc_config, model));
 printf("%zu %zu %zu %zu\n", sizeof(cumc_batch_config), offsetof(cumc_batch_config, t_end),
 offsetof(cumc_batch_config, cfl), offsetof(cumc_batch_config, positivity_fallback));return 0;}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    assert vals == [C.sizeof(capi.CumcModel), C.sizeof(capi.CumcConfig), capi.CumcConfig.xF.offset,
                    capi.CumcConfig.cfl.offset, capi.CumcConfig.model.offset,
                    C.sizeof(capi.CumcBatchConfig), capi.CumcBatchConfig.t_end.offset,
                    capi.CumcBatchConfig.cfl.offset, capi.CumcBatchConfig.positivity_fallback.offset]


def test_create_rejects_bad_configs_before_touching_the_device():
    from cumc3d_b200 import models
    L = engine.load_library()
    spec, _, _ = models.blast_3d(8)
    spec["boundary_flag"] = [0, 1, 0, 0, 0, 0]  # unpaired periodic
    cfg, keep = capi.make_config(spec)
    h = C.c_void_p()
    assert L.cumc_create(C.byref(cfg), C.byref(h)) == capi.CUMC_EINVAL
    assert b"pairs" in L.cumc_last_error(None)
    spec["boundary_flag"] = [4, 4, 0, 0, 0, 0]  # equatorial symmetry on x: setup.f90:119-121
    cfg, keep = capi.make_config(spec)
    rc = L.cumc_create(C.byref(cfg), C.byref(h))
    assert rc in (capi.CUMC_EINVAL, capi.CUMC_ECUDA)


def test_no_cpu_fallback_without_device():
    """Without a CUDA device the engine refuses to run (no silent CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cumc3d_b200 import models
    spec, _, _ = models.brio_wu(32)
    with pytest.raises(engine.CumcError) as e:
        engine.Solver(spec)
    assert e.value.code == capi.CUMC_ECUDA


def test_header_is_strict_c99_and_links_every_function():
    """A C host: the header compiles as ISO C99 with every warning an error,
    and a program that takes the address of every declared function links
    against the engine library (nothing is run: no device is needed)."""
    import tempfile
    funcs = declared_functions()
    body = "\n".join("    (void)&%s;" % f for f in funcs)
    src = '#include "cumc3d_gpu.h"\nint main(void) {\n%s\n    return 0;\n}\n' % body
    lib = engine.LIB_PATH
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "all.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "all")
        r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                            os.path.join(ROOT, "include"), c, lib, "-Wl,--allow-shlib-undefined", "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    assert len(funcs) > 50


def test_train_config_layout_matches_header():
    import tempfile
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "cumc3d_gpu.h"
int main(void){printf("%zu %zu %zu\n", sizeof(cumc_train_config), offsetof(cumc_train_config, lr),
 offsetof(cumc_train_config, seed));return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    assert vals == [C.sizeof(capi.CumcTrainConfig), capi.CumcTrainConfig.lr.offset, capi.CumcTrainConfig.seed.offset]
