"""Exact FP64 operation counts per zone-update of the benchmark workloads,
from the oracle built on its counting scalar type (every +, -, *, /, sqrt
and comparison of the restated Fortran counted; test and measurement
infrastructure, not part of the engine).

    python oracle/count_ops.py            # writes profiles/op_counts.json

A zone-update is one zone through one SSP-RK3 step (three stages) plus the
step's FINDDT.  Each workload is counted on two grids of the same initial
state, the second with twice the cells per axis; the per-zone count is
c(s) = A + B / s (the faces and ghost layers add a surface term), so the
large-grid count is A = 2 c(2) - c(1).  Counts split by phase: "recon"
(face reconstruction), "riemann" (BUILDSTATES + the Riemann solver),
"finddt", "other" (CT, source terms, RK combination, recovery, floors,
boundaries).  "flops" counts add, mul, div and sqrt as one each (a
division or square root is many FP64 instructions on the GPU; the
comparisons are listed apart).  The branches of HLLD and of the limiters
depend on the state, so the counts are those of the first step of each
workload's initial state.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from cumc3d_b200 import models  # noqa: E402
from oracle import oracle as O  # noqa: E402

OPS = ("add", "mul", "div", "sqrt", "cmp")
PHASES = ("recon", "riemann", "finddt", "other")


def _blast(n):
    spec, prim, eps = models.blast_3d(n, recon="weno", riemann="hlld")
    spec["positivity_fallback"] = 1
    spec["fix_periodic_normal_faces"] = 1
    return spec, prim, eps


# name -> (builder of the grid at scale s, scales, directions swept)
WORKLOADS = {
    "blast3d_weno_hlld": (lambda s: _blast(16 * s), (1, 2), 3),
    "alfven3d_weno_hlld": (lambda s: models.alfven_3d(16 * s, recon="weno"), (1, 2), 3),
    "alfven3d_ppm_hlld": (lambda s: models.alfven_3d(16 * s, recon="ppm"), (1, 2), 3),
    "torus_cyl_weno_hlld": (lambda s: models.torus_cyl(nr=24 * s, nphi=16 * s, nz=24 * s), (1, 2), 3),
    "briowu_ppm_hlld": (lambda s: models.brio_wu(400 * s), (1, 2), 1),
}


def count_one(build):
    spec, prim, eps = build()
    zones = spec["nx"] * spec["ny"] * spec["nz"]
    o = O.Oracle(spec, counting=True)
    o.set_state(prim, eps)
    o.initial_update()
    O.reset_counts()
    dt = o.finddt()
    o.rk3_step(dt)
    out = {ph: {k: v / zones for k, v in O.get_counts(ph).items()} for ph in PHASES}
    o.close()
    return out, zones


def main():
    O.build()
    result = {}
    for name, (build, scales, ndir) in WORKLOADS.items():
        t0 = time.time()
        per = {}
        for s in scales:
            per[s], zones = count_one(lambda s=s: build(s))
            per[s]["zones"] = zones
        c1, c2 = per[scales[0]], per[scales[1]]
        ext = {ph: {k: 2 * c2[ph][k] - c1[ph][k] for k in OPS} for ph in PHASES}

        def flops(c):
            return sum(c[k] for k in ("add", "mul", "div", "sqrt"))
        total = {k: sum(ext[ph][k] for ph in PHASES) for k in OPS}
        result[name] = {
            "per_zone_update": ext,
            "total": total,
            "flops_per_zone_update": flops(total),
            # one reconstruction + Riemann sweep (the face-flux kernel pair)
            # of one stage in one direction, per zone
            "flux_sweep_flops_per_zone": (flops(ext["recon"]) + flops(ext["riemann"])) / (3 * ndir),
            "samples": {str(per[s]["zones"]): {"flops_per_zone_update": sum(flops(per[s][ph]) for ph in PHASES)}
                        for s in scales},
        }
        print(name, "%.0f flops/zone-update" % result[name]["flops_per_zone_update"],
              "(%.1f s)" % (time.time() - t0), flush=True)
    result["_command"] = "python oracle/count_ops.py"
    with open(os.path.join(ROOT, "profiles", "op_counts.json"), "w") as f:
        json.dump(result, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
