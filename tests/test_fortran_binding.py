"""The Fortran binding (CPU): cumc3d_b200/fortran/cumc_gpu.f90 cannot be
compiled here (no Fortran compiler), so this checks it against the C header
as text: every function include/cumc3d_gpu.h declares has an interface
bound to that exact name, with one dummy argument per C parameter, and every
#define constant the module repeats has the header's value."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header():
    with open(os.path.join(ROOT, "include", "cumc3d_gpu.h")) as f:
        h = f.read()
    h = re.sub(r"/\*.*?\*/", " ", h, flags=re.S)
    funcs = {}
    for m in re.finditer(r"^[ \t]*(?:const[ \t]+)?[A-Za-z_][A-Za-z0-9_]*[ \t\*]+(cumc_[a-z0-9_]+)[ \t]*\(([^)]*)\)\s*;",
                         h, re.M):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        funcs[m.group(1)] = len(args)
    defines = dict(re.findall(r"^#define[ \t]+(CUMC_[A-Z0-9_]+)[ \t]+(-?\d+)", h, re.M))
    return funcs, defines


def _module():
    with open(os.path.join(ROOT, "cumc3d_b200", "fortran", "cumc_gpu.f90")) as f:
        src = f.read()
    src = re.sub(r"&[ \t]*\n[ \t]*", " ", src)               # join continuation lines
    src = re.sub(r"!.*", "", src)                             # drop comments
    funcs = {}
    for m in re.finditer(r"FUNCTION[ \t]+(\w+)[ \t]*\(([^)]*)\)[ \t]*BIND\(C,[ \t]*NAME='(cumc_[a-z0-9_]+)'\)", src):
        funcs[m.group(3)] = len([a for a in m.group(2).split(",") if a.strip()])
    params = {}
    for decl in re.findall(r"PARAMETER[ \t]*::[ \t]*(.*)", src):
        for name, val in re.findall(r"(CUMC_[A-Z0-9_]+)[ \t]*=[ \t]*(-?\d+)", decl):
            params[name] = val
    return funcs, params


def test_every_entry_point_is_bound_with_its_arity():
    hf, _ = _header()
    mf, _ = _module()
    assert len(hf) > 50
    missing = sorted(set(hf) - set(mf))
    assert not missing, missing
    assert not sorted(set(mf) - set(hf))
    wrong = {n: (hf[n], mf[n]) for n in hf if hf[n] != mf[n]}
    assert not wrong, wrong


def test_constants_repeat_the_header_values():
    _, hd = _header()
    _, mp = _module()
    shared = set(hd) & set(mp)
    assert len(shared) > 20
    assert {k: (hd[k], mp[k]) for k in shared if hd[k] != mp[k]} == {}
