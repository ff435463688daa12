"""Initial models (the reference's GET_MODEL hooks) and named workloads.

Each builder returns ``(spec, prim, eps)``:

* ``spec`` -- a dict that :func:`cumc3d_b200.capi.make_config` turns into a
  ``cumc_config`` (grid, flags, solver options, model descriptor);
* ``prim`` -- float64 array of shape (nz+6, ny+6, nx+6, 8), the Fortran
  ``prim(1:8,-2:nx+3,-2:ny+3,-2:nz+3)`` in memory order;
* ``eps``  -- float64 array of shape (nz+6, ny+6, nx+6).

Cells the reference's GET_MODEL leaves unset hold NaN in ``eps`` (its
``epsilon`` array is never zeroed, solver/mhd/initial.f90:68-70 only zeroes
``prim`` and ``cons``), so any read of an undefined value becomes visible.
"""
import math

import numpy as np

from .capi import IBX, IBY, IBZ, IRHO, ITAU, IVX, IVY, IVZ


def faces(start, end, n):
    """Uniform face coordinates for indices -3..n+3 (solver/mhd/getgrid.f90:26-34)."""
    d = (end - start) / float(n)
    j = np.arange(-3, n + 4, dtype=np.float64)
    return start + j * d


def centers(xf):
    """Cell centres for indices -2..n+3 (solver/mhd/getgrid.f90:55-63)."""
    return (xf[1:] + xf[:-1]) / 2.0


def _alloc(nx, ny, nz):
    prim = np.zeros((nz + 6, ny + 6, nx + 6, 8), dtype=np.float64)
    eps = np.full((nz + 6, ny + 6, nx + 6), np.nan, dtype=np.float64)
    return prim, eps


def _base_spec(nx, ny, nz, n_dim, bflag, xr, yr, zr, **kw):
    spec = dict(nx=nx, ny=ny, nz=nz, n_dim=n_dim, coordinate_flag=kw.pop("coordinate_flag", 0),
                boundary_flag=list(bflag),
                xF=faces(xr[0], xr[1], nx), yF=faces(yr[0], yr[1], ny), zF=faces(zr[0], zr[1], nz))
    spec.update(kw)
    return spec


# ---------------------------------------------------------------------------
# 1D Brio-Wu shock tube: model/riemann/src/riemann1d.f90:229-250 (test 10)
# ---------------------------------------------------------------------------
def brio_wu(nx=800, recon="ppm", riemann="hlld", cfl=0.8, precision="fp64"):
    spec = _base_spec(nx, 1, 1, 1, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), (0.0, 1.0),
                      cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      model=dict(gamma=2.0, floor="eps"), t_end=0.1,
                      name="brio_wu_%d" % nx)
    prim, eps = _alloc(nx, 1, 1)
    g = 2.0
    x = centers(spec["xF"])  # index -2..nx+3 -> position j+2
    for j in range(0, nx + 1):
        left = x[j + 2] <= 0.5
        prim[:, :, j + 2, IRHO] = 1.0 if left else 0.125
        prim[:, :, j + 2, ITAU] = 1.0 if left else 0.1
        prim[:, :, j + 2, IBY] = 1.0 if left else -1.0
        prim[:, :, j + 2, IBX] = 0.75
        eps[:, :, j + 2] = prim[:, :, j + 2, ITAU] / prim[:, :, j + 2, IRHO] / (g - 1.0)
    return spec, prim, eps


# ---------------------------------------------------------------------------
# 1D Riemann problem with arbitrary left/right states (the batched workload)
# ---------------------------------------------------------------------------
def riemann_1d(nx, left, right, bx, gamma=5.0 / 3.0, recon="ppm", riemann="hlld", cfl=0.8,
               precision="fp64", t_end=0.1):
    """left/right: dicts with rho, p, vx, vy, vz, by, bz.  Bx shared by both sides."""
    spec = _base_spec(nx, 1, 1, 1, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), (0.0, 1.0),
                      cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      model=dict(gamma=gamma, floor="eps"), t_end=t_end, name="riemann1d_%d" % nx)
    prim, eps = _alloc(nx, 1, 1)
    x = centers(spec["xF"])
    for j in range(0, nx + 1):
        s = left if x[j + 2] <= 0.5 else right
        prim[:, :, j + 2, IRHO] = s["rho"]
        prim[:, :, j + 2, ITAU] = s["p"]
        prim[:, :, j + 2, IVX] = s["vx"]
        prim[:, :, j + 2, IVY] = s["vy"]
        prim[:, :, j + 2, IVZ] = s["vz"]
        prim[:, :, j + 2, IBY] = s["by"]
        prim[:, :, j + 2, IBZ] = s["bz"]
        prim[:, :, j + 2, IBX] = bx
        eps[:, :, j + 2] = s["p"] / s["rho"] / (gamma - 1.0)
    return spec, prim, eps


# ---------------------------------------------------------------------------
# the riemann model's 1D set: model/riemann/src/riemann1d.f90:28-330
# ---------------------------------------------------------------------------
_S4PI = 1.0 / math.sqrt(4.0 * math.pi)
RIEMANN_1D = {
    # test_model: (name, gamma, boundary_flag, t_end, left, right); a state
    # is {var: value}, split at x = 0.5 unless the test says otherwise
    1: ("toro1", 1.4, (1, 1, 1, 1, 1, 1), 0.25, {IRHO: 1.0, ITAU: 1.0}, {IRHO: 0.125, ITAU: 0.1}),
    2: ("toro2", 1.4, (1, 1, 1, 1, 1, 1), 0.15, {IVX: -2.0, IRHO: 1.0, ITAU: 0.4}, {IVX: 2.0, IRHO: 1.0, ITAU: 0.4}),
    3: ("toro3", 1.4, (1, 1, 1, 1, 1, 1), 0.012, {ITAU: 1000.0, IRHO: 1.0}, {ITAU: 0.01, IRHO: 1.0}),
    4: ("toro4", 1.4, (1, 1, 1, 1, 1, 1), 0.035, {ITAU: 0.01, IRHO: 1.0}, {ITAU: 100.0, IRHO: 1.0}),
    5: ("toro5", 1.4, (1, 1, 1, 1, 1, 1), 0.035, {IVX: 19.5975, ITAU: 460.894, IRHO: 5.99924},
        {IVX: -6.19633, ITAU: 46.0950, IRHO: 5.99924}),
    6: ("interacting_shocks", 1.4, (2, 2, 1, 1, 1, 1), 0.038, None, None),
    7: ("shu_osher", 1.4, (1, 1, 1, 1, 1, 1), 0.178, None, None),
    8: ("sedov", 1.4, (2, 1, 1, 1, 1, 1), 0.47, None, None),
    9: ("dai_woodward", 5.0 / 3.0, (1, 1, 1, 1, 1, 1), 0.15, {IRHO: 1.0, ITAU: 1.0, IBY: 1.0, IBX: 1.0},
        {IRHO: 0.2, ITAU: 0.1, IBY: 0.0, IBX: 1.0}),
    10: ("brio_wu", 2.0, (1, 1, 1, 1, 1, 1), 0.1, {IRHO: 1.0, ITAU: 1.0, IBY: 1.0, IBX: 0.75},
         {IRHO: 0.125, ITAU: 0.1, IBY: -1.0, IBX: 0.75}),
    11: ("seven_discontinuities", 5.0 / 3.0, (1, 1, 1, 1, 1, 1), 0.2,
         {IRHO: 1.08, ITAU: 0.95, IVX: 1.2, IVY: 0.01, IVZ: 0.5, IBY: 3.6 * _S4PI, IBX: 2.0 * _S4PI, IBZ: 2.0 * _S4PI},
         {IRHO: 1.0, ITAU: 1.0, IVX: 0.0, IVY: 0.0, IVZ: 0.0, IBY: 4.0 * _S4PI, IBX: 2.0 * _S4PI, IBZ: 2.0 * _S4PI}),
    12: ("magnetosonic_rarefactions", 5.0 / 3.0, (1, 1, 1, 1, 1, 1), 0.1,
         {IVX: -1.0, IRHO: 1.0, ITAU: 1.0, IBY: 1.0}, {IVX: 1.0, IRHO: 1.0, ITAU: 1.0, IBY: 1.0}),
    13: ("two_fast_shocks", 5.0 / 3.0, (1, 1, 1, 1, 1, 1), 0.03,
         {IVX: 36.87, IVY: -0.155, IVZ: -0.0386, IRHO: 1.0, ITAU: 1.0, IBX: 4.0 * _S4PI, IBY: 4.0 * _S4PI,
          IBZ: 1.0 * _S4PI},
         {IVX: -36.87, IVY: 0.0, IVZ: 0.0, IRHO: 1.0, ITAU: 1.0, IBX: 4.0 * _S4PI, IBY: 4.0 * _S4PI,
          IBZ: 1.0 * _S4PI}),
}


def riemann_1d_test(test_model, nx=800, recon="ppm", riemann="hlld", cfl=0.8, precision="fp64"):
    """The riemann model's 1D tests by test_model number (riemann1d.f90:
    1-5 Toro's tests, 6 two interacting blast waves (reflecting), 7
    Shu-Osher, 8 Sedov (reflecting inner side, Cartesian: mu = 1), 9 Dai &
    Woodward, 10 Brio-Wu, 11 seven discontinuities, 12 magnetosonic
    rarefactions, 13 two fast shocks) on [0, 1].  As the reference: the
    hydrodynamic tests (1-8) set cells 1..n, the MHD ones (9-13) cells 0..n;
    the rest stays as INITIAL_UPDATE finds it (prim 0, epsilon undefined)."""
    name, g, bflag, t_end, left, right = RIEMANN_1D[test_model]
    spec = _base_spec(nx, 1, 1, 1, bflag, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0), cfl=cfl, recon=recon,
                      riemann=riemann, precision=precision, model=dict(gamma=g, floor="eps"), t_end=t_end,
                      name="riemann1d_%s_%d" % (name, nx))
    prim, eps = _alloc(nx, 1, 1)
    x = centers(spec["xF"])                       # index j+2
    j0 = 0 if test_model >= 9 else 1
    for j in range(j0, nx + 1):
        c = prim[:, :, j + 2]
        xj = x[j + 2]
        if left is not None:
            for v, val in (left if xj <= 0.5 else right).items():
                c[..., v] = val
        elif test_model == 6:
            c[..., ITAU] = 1.0e3 if xj <= 0.1 else (1.0e2 if xj >= 0.9 else 1.0e-2)
            c[..., IRHO] = 1.0
        elif test_model == 7:
            if xj <= 0.1:
                c[..., IRHO], c[..., IVX], c[..., ITAU] = 3.857143, 2.629369, 10.3333
            else:
                c[..., IRHO], c[..., IVX], c[..., ITAU] = 1.0 + 0.2 * math.sin(5.0e1 * xj), 0.0, 1.0
        else:  # 8, Sedov: the blast energy in the first four cells
            mu = 1.0  # coordinate_flag + 1, Cartesian
            c[..., ITAU] = (3.0 * (g - 1.0) * 1.0) / ((1.0 + mu) * math.pi * x[4 + 2] ** mu) if j <= 4 else 1.0e-5
            c[..., IRHO] = 1.0
        eps[:, :, j + 2] = c[..., ITAU] / c[..., IRHO] / (g - 1.0)
    return spec, prim, eps


# ---------------------------------------------------------------------------
# 2D MHD problems of the riemann model: model/riemann/src/riemann2d.f90:441-640
# ---------------------------------------------------------------------------
RIEMANN_2D = {
    # test_model: (name, gamma, boundary_flag, x range, y range, t_end)
    1: ("gresho", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 3.0),
    2: ("toro_blast", 1.4, (2, 2, 2, 2, 1, 1), (0.0, 1.0), (0.0, 1.5), 1.0),
    3: ("toro_explosion", 1.4, (2, 1, 2, 1, 1, 1), (0.0, 1.5), (0.0, 1.5), 2.667),
    4: ("implosion", 1.4, (2, 2, 2, 2, 1, 1), (0.0, 0.3), (0.0, 0.3), 2.5),
    5: ("kelvin_helmholtz_hydro", 1.4, (0, 0, 0, 0, 1, 1), (0.0, 1.0), (0.0, 1.0), 5.0),
    6: ("rayleigh_taylor_hydro", 1.4, (0, 0, 2, 2, 1, 1), (0.0, 0.5), (0.0, 1.5), 12.75),
    7: ("quadrants_3", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.3),
    8: ("quadrants_4", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.25),
    9: ("quadrants_6", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.3),
    10: ("quadrants_12", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.25),
    11: ("quadrants_15", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.2),
    12: ("quadrants_17", 1.4, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.3),
    13: ("current_sheet", 5.0 / 3.0, (0, 0, 0, 0, 1, 1), (0.0, 1.0), (0.0, 1.0), 10.0),
    14: ("rotor", 5.0 / 3.0, (1, 1, 1, 1, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.295),
    15: ("orszag_tang", 5.0 / 3.0, (0, 0, 0, 0, 1, 1), (0.0, 1.0), (0.0, 1.0), 1.0),
    16: ("blast", 5.0 / 3.0, (0, 0, 0, 0, 1, 1), (0.0, 1.0), (0.0, 1.0), 0.2),
    17: ("kelvin_helmholtz", 1.4, (0, 0, 0, 0, 1, 1), (0.0, 1.0), (0.0, 1.0), 5.0),
    18: ("rayleigh_taylor", 1.4, (0, 0, 2, 2, 1, 1), (0.0, 1.0), (0.0, 1.0), 12.5),
    19: ("current_loop", 5.0 / 3.0, (0, 0, 0, 0, 1, 1), (-1.0, 1.0), (-0.5, 0.5), 2.0),
}


# the four-quadrant problems (tests 7-12): (rho, p, vx, vy) in the quadrants
# (x < 0.5, y < 0.5), (x > 0.5, y < 0.5), (x < 0.5, y > 0.5), (x > 0.5, y > 0.5)
_QUADRANTS = {
    7: ((0.138, 0.0290, 1.2060, 1.2060), (0.5323, 0.3, 0.0, 1.2060), (0.5323, 0.3, 1.2060, 0.0), (1.5, 1.5, 0.0, 0.0)),
    8: ((1.1, 1.1, 0.8939, 0.8939), (0.5065, 0.35, 0.0, 0.8939), (0.5065, 0.35, 0.8939, 0.0), (1.1, 1.1, 0.0, 0.0)),
    9: ((1.0, 1.0, -0.75, 0.5), (3.0, 1.0, -0.75, -0.5), (2.0, 1.0, 0.75, 0.5), (1.0, 1.0, 0.75, -0.5)),
    10: ((0.8, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.7276), (1.0, 1.0, 0.7276, 0.5), (0.5313, 0.4, 0.0, 0.0)),
    11: ((0.8, 0.4, 0.1, -0.3), (0.5313, 0.4, 0.1, 0.4276), (0.5197, 0.4, -0.6259, -0.3), (1.0, 1.0, 0.1, -0.3)),
    12: ((1.0625, 0.4, 0.0, 0.2145), (0.5197, 0.4, 0.0, -1.1259), (2.0, 1.0, 0.0, -0.3), (1.0, 1.0, 0.0, -0.4)),
}


def riemann_2d(test_model, nx=128, ny=None, recon="ppm", riemann="hlld", cfl=0.4, precision="fp64", seed=20261203):
    """The riemann model's 2D set by its test_model number (riemann2d.f90):
    hydrodynamics -- 1 Gresho vortex, 2 Toro's blast, 3 Toro's explosion
    (Cartesian), 4 implosion, 5 Kelvin-Helmholtz, 6 Rayleigh-Taylor, 7-12
    the four-quadrant Riemann problems (configurations 3, 4, 6, 12, 15, 17);
    MHD (riemann2d.f90:441-640) -- 13 current sheet, 14 rotor, 15
    Orszag-Tang vortex, 16 blast, 17 Kelvin-Helmholtz, 18 Rayleigh-Taylor, 19
    advected current loop.  Both Rayleigh-Taylor tests feel the model's
    constant gravity g = 0.1 in -y (custom.f90:132-159).  Boundaries, boxes,
    gamma and end times as the file states them; as the reference, the
    hydrodynamic tests set cells 1..n and the MHD ones 0..n, face fields from
    the cell-centre formulas as the reference writes them, the loop's from a
    corner vector potential.  The seeded uniform numbers stand in for
    RANDOM_NUMBER (5, 17, 18)."""
    name, g, bflag, xr, yr, t_end = RIEMANN_2D[test_model]
    ny = ny or nx
    model = dict(gamma=g, floor="eps")
    if test_model in (6, 18):
        model.update(source="const_gy", g_const=0.1)
    spec = _base_spec(nx, ny, 1, 2, bflag, xr, yr, (0.0, 1.0), cfl=cfl, recon=recon, riemann=riemann,
                      precision=precision, model=model, t_end=t_end, name="riemann2d_%s_%dx%d" % (name, nx, ny))
    prim, eps = _alloc(nx, ny, 1)
    x, y = centers(spec["xF"]), centers(spec["yF"])
    xF, yF = spec["xF"][1:], spec["yF"][1:]           # xF(j) at index j+2
    dx, dy = spec["xF"][1:] - spec["xF"][:-1], spec["yF"][1:] - spec["yF"][:-1]
    lo = 2 if test_model >= 13 else 3                   # first cell set: 0 (MHD) or 1
    J, K = slice(lo, nx + 3), slice(lo, ny + 3)
    X, Y = np.meshgrid(x[J], y[K], indexing="xy")      # [k, j]
    P = np.zeros(X.shape + (8,))
    rng = np.random.Generator(np.random.PCG64(seed))
    pi = math.pi
    if test_model == 1:
        d = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
        ds = np.where(d > 0.0, d, 1.0)
        inner, ring = d <= 0.2, (d > 0.2) & (d <= 0.4)
        P[..., ITAU] = np.where(inner, 5.0 + 12.5 * d ** 2,
                                np.where(ring, 9.0 - 4.0 * math.log(0.2) + 12.5 * d ** 2 - 20.0 * d
                                         + 4.0 * np.log(np.where(ring, d, 1.0)), 3.0 + 4.0 * math.log(2.0)))
        P[..., IVX] = np.where(inner, -5.0 * (Y - 0.5), np.where(ring, -(2.0 - 5.0 * d) * (Y - 0.5) / ds, 0.0))
        P[..., IVY] = np.where(inner, 5.0 * (X - 0.5), np.where(ring, (2.0 - 5.0 * d) * (X - 0.5) / ds, 0.0))
        P[..., IRHO] = 1.0
    elif test_model == 2:
        d = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
        P[..., ITAU] = np.where(d <= 0.1, 10.0, 1.0)
        P[..., IRHO] = 1.0
    elif test_model == 3:
        inside = np.sqrt(X ** 2 + Y ** 2) < 0.4
        P[..., IRHO] = np.where(inside, 1.0, 0.125)
        P[..., ITAU] = np.where(inside, 1.0, 0.1)
    elif test_model == 4:
        outer = X + Y > 0.15
        P[..., IRHO] = np.where(outer, 1.0, 0.125)
        P[..., ITAU] = np.where(outer, 1.0, 0.14)
    elif test_model == 5:
        outer = (Y > 0.75) | (Y < 0.25)
        d = rng.random(X.shape + (2,))                  # two draws per cell, in loop order
        P[..., IRHO] = np.where(outer, 1.0, 2.0)
        P[..., IVX] = np.where(outer, -0.5 + 0.01 * (d[..., 0] - 0.5), 0.5 + 0.01 * (d[..., 0] - 0.5))
        P[..., IVY] = 0.01 * (d[..., 1] - 0.5)
        P[..., ITAU] = 2.5
    elif test_model == 6:
        P[..., IRHO] = np.where(Y < 0.75, 1.0, 2.0)
        P[..., ITAU] = 2.5 - 0.1 * P[..., IRHO] * Y
        P[..., IVY] = 0.025 * (1.0 + np.cos(4.0 * pi * (X - 0.25))) * (1.0 + np.cos(3.0 * pi * (Y - 0.75)))
    elif test_model <= 12:
        xl, xh = (X > 0.0) & (X < 0.5), (X > 0.5) & (X < 1.0)
        yl, yh = (Y > 0.0) & (Y < 0.5), (Y > 0.5) & (Y < 1.0)
        for q, m in zip(_QUADRANTS[test_model], (xl & yl, xh & yl, xl & yh, xh & yh)):
            for v, val in zip((IRHO, ITAU, IVX, IVY), q):
                P[..., v] = np.where(m, val, P[..., v])
    elif test_model == 13:
        P[..., IBY] = np.where((X <= 0.25) | (X >= 0.75), 1.0, -1.0) / math.sqrt(4.0 * pi)
        P[..., IRHO] = 1.0
        P[..., ITAU] = 0.1 * 0.5
        P[..., IVX] = 0.1 * np.sin(2.0 * pi * (Y - 0.5))
    elif test_model == 14:
        r0, r1 = 0.1, 0.115
        r = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
        fr = (r1 - r) / (r1 - r0)
        inner, outer = r <= r0, r >= r1
        rs = np.where(inner | outer, 1.0, r)
        P[..., IRHO] = np.where(inner, 10.0, np.where(outer, 1.0, 1.0 + 9.0 * fr))
        P[..., IVX] = np.where(inner, -1.0 * (Y - 0.5) / r0, np.where(outer, 0.0, -fr * 1.0 * (Y - 0.5) / rs))
        P[..., IVY] = np.where(inner, 1.0 * (X - 0.5) / r0, np.where(outer, 0.0, fr * 1.0 * (X - 0.5) / rs))
        P[..., ITAU] = 0.5
        P[..., IBX] = 2.5 / math.sqrt(4.0 * pi)
    elif test_model == 15:
        P[..., IRHO] = 25.0 / 36.0 / pi
        P[..., ITAU] = 5.0 / 12.0 / pi
        P[..., IVX] = -np.sin(2.0 * pi * Y)
        P[..., IVY] = np.sin(2.0 * pi * X)
        P[..., IBX] = -np.sin(2.0 * pi * Y) / math.sqrt(4.0 * pi)
        P[..., IBY] = np.sin(4.0 * pi * X) / math.sqrt(4.0 * pi)
    elif test_model == 16:
        d = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
        P[..., ITAU] = np.where(d <= 0.1, 10.0, 0.1)
        P[..., IRHO] = 1.0
        P[..., IBX] = 1.0 / math.sqrt(2)
        P[..., IBY] = 1.0 / math.sqrt(2)
    elif test_model == 17:
        outer = (Y > 0.75) | (Y < 0.25)
        d = rng.random(X.shape + (2,))                  # two draws per cell, in loop order
        P[..., IRHO] = np.where(outer, 1.0, 2.0)
        P[..., IVX] = np.where(outer, 0.5 + 0.01 * d[..., 0], -0.5 + 0.01 * d[..., 0])
        P[..., ITAU] = 2.5
        P[..., IVY] = 0.01 * d[..., 1]
        P[..., IBX] = 0.2
    elif test_model == 18:
        P[..., IRHO] = np.where(Y <= 0.5, 1.0, 2.0)
        P[..., ITAU] = 2.5 - 0.1 * P[..., IRHO] * (Y - 0.5)
        d = rng.random(X.shape)
        P[..., IVY] = 0.01 * d * (1.0 + np.cos(8.0 * pi * (Y - 0.5) / 3.0)) / 2.0
        P[..., IBX] = 0.0125
    else:  # 19: face field from the corner vector potential (cells 0..n)
        P[..., IRHO] = 1.0
        P[..., ITAU] = 1.0
        P[..., IVX] = 2.0
        P[..., IVY] = 1.0
        XF, YF = np.meshgrid(xF[J], yF[K], indexing="xy")
        a = np.zeros((ny + 2, nx + 2))                  # corners -1..n, zero at -1
        a[1:, 1:] = 0.001 * np.maximum(0.0, 0.3 - np.sqrt(XF ** 2 + YF ** 2))
        P[..., IBX] = (a[1:, 1:] - a[:-1, 1:]) / dy[K][:, None]
        P[..., IBY] = -(a[1:, 1:] - a[1:, :-1]) / dx[J][None, :]
    prim[:, K, J, :] = P[None]
    with np.errstate(divide="ignore", invalid="ignore"):
        eps[:, K, J] = (P[..., ITAU] / P[..., IRHO] / (g - 1.0))[None]
    return spec, prim, eps


def riemann_3d(test_model, n=64, recon="ppm", riemann="hlld", cfl=0.4, precision="fp64"):
    """The riemann model's 3D set (model/riemann/src/riemann3d.f90): 1 the
    spherical explosion in the unit cube (rho, p = 1 inside r < 0.4 of the
    origin corner, 0.125, 0.1 outside; gamma 1.4; the boundary flags its
    comment gives, (1,2,1,2,1,2)), 2 the oblique Sod tube (bands of x+y+z
    at 0.5, 1, 1.5; gamma 5/3; outflow).  Cells 1..n set, as the reference."""
    if test_model == 1:
        g, bflag, name = 1.4, (1, 2, 1, 2, 1, 2), "explosion"
    elif test_model == 2:
        g, bflag, name = 5.0 / 3.0, (1, 1, 1, 1, 1, 1), "oblique_sod"
    else:
        raise ValueError("no such test model")
    spec = _base_spec(n, n, n, 3, bflag, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0), cfl=cfl, recon=recon,
                      riemann=riemann, precision=precision, model=dict(gamma=g, floor="eps"),
                      name="riemann3d_%s_%d" % (name, n))
    prim, eps = _alloc(n, n, n)
    c = centers(spec["xF"])[3:n + 3]
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    P = np.zeros(X.shape + (8,))
    if test_model == 1:
        inside = np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < 0.4
        P[..., IRHO] = np.where(inside, 1.0, 0.125)
        P[..., ITAU] = np.where(inside, 1.0, 0.1)
    else:
        s = X + Y + Z
        band = (s < 0.5) | ((s > 1.0) & (s < 1.5))
        P[..., IRHO] = np.where(band, 4.0, 1.0)
        P[..., ITAU] = np.where(band, 1.0, 0.1795)
    prim[3:n + 3, 3:n + 3, 3:n + 3] = P
    eps[3:n + 3, 3:n + 3, 3:n + 3] = P[..., ITAU] / P[..., IRHO] / (g - 1.0)
    return spec, prim, eps


def batch_problems(n_problems=512, seed=20261203, nmin=128, nmax=4096):
    """Seeded parameters of the batched workload (one 1D Riemann problem each)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n_problems):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        sides = []
        for _s in range(2):
            sides.append(dict(
                rho=float(math.exp(rng.uniform(math.log(0.1), math.log(10.0)))),
                p=float(math.exp(rng.uniform(math.log(0.01), math.log(10.0)))),
                vx=float(rng.uniform(-1, 1)), vy=float(rng.uniform(-1, 1)), vz=float(rng.uniform(-1, 1)),
                by=float(rng.uniform(-2, 2)), bz=float(rng.uniform(-2, 2))))
        bx = float(rng.uniform(-1, 1))
        out.append(dict(n=n, left=sides[0], right=sides[1], bx=bx))
    return out


# ---------------------------------------------------------------------------
# 3D MHD blast: the 3D analogue of model/riemann/src/riemann2d.f90:522-544
# ---------------------------------------------------------------------------
def blast_3d(n=256, recon="weno", riemann="hlld", cfl=0.4, precision="fp64", nx=None, ny=None, nz=None,
             radius=0.1, p_in=10.0, p_out=0.1):
    nx = nx or n
    ny = ny or n
    nz = nz or n
    spec = _base_spec(nx, ny, nz, 3, (0, 0, 0, 0, 0, 0), (-0.5, 0.5), (-0.5, 0.5), (-0.5, 0.5),
                      cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      model=dict(gamma=5.0 / 3.0, floor="eps"), steps=200,
                      name="blast3d_%dx%dx%d" % (nx, ny, nz))
    g = 5.0 / 3.0
    x = centers(spec["xF"])
    y = centers(spec["yF"])
    z = centers(spec["zF"])
    r = np.sqrt(z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2)
    prim = np.zeros((nz + 6, ny + 6, nx + 6, 8), dtype=np.float64)
    prim[..., IRHO] = 1.0
    prim[..., ITAU] = np.where(r <= radius, p_in, p_out)
    b0 = 1.0 / math.sqrt(2.0)
    prim[..., IBX] = b0
    prim[..., IBY] = b0
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    return spec, prim, np.ascontiguousarray(eps)


# ---------------------------------------------------------------------------
# 3D circularly polarised Alfven wave along (1,1,1)/sqrt(3)
# ---------------------------------------------------------------------------
def alfven_3d(n=256, recon="ppm", riemann="hlld", cfl=0.4, precision="fp64", amp=0.1,
              fix_periodic_normal_faces=1):
    """Face B from an edge-centred vector potential, so div B = 0 to roundoff.

    Wave vector k = 2*pi*(1,1,1) on the unit periodic box (wavelength 1/sqrt3).
    B = B_par e1 + amp (cos(phase) e2 + sin(phase) e3), v = -amp/sqrt(rho) (...)
    with e1 = (1,1,1)/sqrt3 the propagation direction.
    """
    spec = _base_spec(n, n, n, 3, (0, 0, 0, 0, 0, 0), (0.0, 1.0), (0.0, 1.0), (0.0, 1.0),
                      cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      fix_periodic_normal_faces=fix_periodic_normal_faces,
                      model=dict(gamma=5.0 / 3.0, floor="eps"), name="alfven3d_%d" % n)
    g = 5.0 / 3.0
    rho0, p0, bpar = 1.0, 0.1, 1.0
    kk = 2.0 * math.pi
    e1 = np.array([1.0, 1.0, 1.0]) / math.sqrt(3.0)
    e2 = np.array([1.0, -1.0, 0.0]) / math.sqrt(2.0)
    e3 = np.cross(e1, e2)
    xF, yF, zF = spec["xF"], spec["yF"], spec["zF"]
    xc, yc, zc = centers(xF), centers(yF), centers(zF)
    kvec = kk * np.array([1.0, 1.0, 1.0])
    kmag = np.linalg.norm(kvec)

    # vector potential A = B_par/2 (e1 x r) - amp/|k| (cos(phase) e2 + sin(phase) e3):
    # curl of f(phase) w is k x f'(phase) w, and e1 x e2 = e3, e1 x e3 = -e2, so
    # curl A = B_par e1 + amp (cos(phase) e2 + sin(phase) e3), the same transverse
    # field the velocity below is built from (an exact travelling Alfven wave)
    def A(px, py, pz):
        phase = kvec[0] * px + kvec[1] * py + kvec[2] * pz
        r = np.stack(np.broadcast_arrays(px, py, pz), axis=-1)
        uni = 0.5 * bpar * np.cross(e1, r)
        wav = -(amp / kmag) * (np.cos(phase)[..., None] * e2 + np.sin(phase)[..., None] * e3)
        return uni + wav

    prim = np.zeros((n + 6, n + 6, n + 6, 8), dtype=np.float64)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    phase = kvec[0] * X + kvec[1] * Y + kvec[2] * Z
    bperp = amp * (np.cos(phase)[..., None] * e2 + np.sin(phase)[..., None] * e3)
    vperp = -bperp / math.sqrt(rho0)
    prim[..., IRHO] = rho0
    prim[..., ITAU] = p0
    prim[..., IVX] = vperp[..., 0]
    prim[..., IVY] = vperp[..., 1]
    prim[..., IVZ] = vperp[..., 2]
    # face B = (1/area) * circulation of A around the face (edge midpoints, Stokes)
    # x-face at (xF[j], y-center, z-center): Bx = (Az(y+)-Az(y-))/dy - (Ay(z+)-Ay(z-))/dz
    dy = yF[1:] - yF[:-1]
    dz = zF[1:] - zF[:-1]
    dx = xF[1:] - xF[:-1]
    ZC, YC, XF = np.meshgrid(zc, yc, xF[1:], indexing="ij")
    Ap = A(XF, YC + 0.5 * dy[None, :, None], ZC)
    Am = A(XF, YC - 0.5 * dy[None, :, None], ZC)
    Bp = A(XF, YC, ZC + 0.5 * dz[:, None, None])
    Bm = A(XF, YC, ZC - 0.5 * dz[:, None, None])
    prim[..., IBX] = (Ap[..., 2] - Am[..., 2]) / dy[None, :, None] - (Bp[..., 1] - Bm[..., 1]) / dz[:, None, None]
    ZC, YF_, XC = np.meshgrid(zc, yF[1:], xc, indexing="ij")
    Ap = A(XC, YF_, ZC + 0.5 * dz[:, None, None])
    Am = A(XC, YF_, ZC - 0.5 * dz[:, None, None])
    Bp = A(XC + 0.5 * dx[None, None, :], YF_, ZC)
    Bm = A(XC - 0.5 * dx[None, None, :], YF_, ZC)
    prim[..., IBY] = (Ap[..., 0] - Am[..., 0]) / dz[:, None, None] - (Bp[..., 2] - Bm[..., 2]) / dx[None, None, :]
    ZF_, YC, XC = np.meshgrid(zF[1:], yc, xc, indexing="ij")
    Ap = A(XC + 0.5 * dx[None, None, :], YC, ZF_)
    Am = A(XC - 0.5 * dx[None, None, :], YC, ZF_)
    Bp = A(XC, YC + 0.5 * dy[None, :, None], ZF_)
    Bm = A(XC, YC - 0.5 * dy[None, :, None], ZF_)
    prim[..., IBZ] = (Ap[..., 1] - Am[..., 1]) / dx[None, None, :] - (Bp[..., 0] - Bm[..., 0]) / dy[None, :, None]
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    vA = bpar / math.sqrt(rho0)
    spec["t_end"] = (1.0 / math.sqrt(3.0)) / vA  # one wave period
    return spec, prim, np.ascontiguousarray(eps)


# ---------------------------------------------------------------------------
# magnetised torus in cylindrical coordinates (model/torus-cyn/src/model.f90)
# ---------------------------------------------------------------------------
def torus_cyl(nr=192, nphi=128, nz=192, r_range=(2.0, 42.0), z_range=(-20.0, 20.0), recon="weno",
              riemann="hlld", cfl=0.4, precision="fp64", learned=0, seed=20261203, s_in=6.0, s_max=10.0,
              rho_atm=1e-6, p_atm=1e-8, rho_cut=0.2, beta_min=100.0, noise=0.01, r_sh=0.0):
    """Constant-angular-momentum (q=2) polytrope, n=1.5, around GM=1.

    Follows GET_MODEL of model/torus-cyn/src/model.f90:6-315 with r_sh=0
    (Newtonian), A_phi proportional to max(rho - rho_cut, 0), the field scaled
    to the minimum plasma beta, and seeded pressure noise.
    """
    g = 5.0 / 3.0
    q = 2.0
    spec = _base_spec(nr, nphi, nz, 3, (1, 1, 0, 0, 1, 1), r_range, (0.0, 2.0 * math.pi), z_range,
                      coordinate_flag=1, cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      learned=learned, steps=2000, name="torus_cyl_%dx%dx%d" % (nr, nphi, nz))
    xF, yF, zF = spec["xF"], spec["yF"], spec["zF"]
    x, z = centers(xF), centers(zF)
    dx = xF[1:] - xF[:-1]
    dz = zF[1:] - zF[:-1]

    def phi_g(r, zz):
        return -1.0 / (np.sqrt(r * r + zz * zz) - r_sh)

    lkep2 = s_max ** (2.0 * q - 1.0) / (s_max - r_sh) ** 2
    c_const = phi_g(s_in, 0.0) - lkep2 * s_in ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q)
    h_max = -phi_g(s_max, 0.0) + lkep2 * s_max ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    k_poly = h_max * (g - 1.0) / g
    R2, Z2 = np.meshgrid(x, z, indexing="xy")  # shape (nz+6, nr+6)
    enth = -phi_g(R2, Z2) + lkep2 * R2 ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    enth = np.maximum(enth, 0.0)
    rho_t = (enth * (g - 1.0) / g / k_poly) ** (1.0 / (g - 1.0))
    inside = (rho_t > rho_atm) & (R2 >= s_in)
    rho2 = np.where(inside, rho_t, rho_atm)
    p2 = np.where(inside, k_poly * rho_t ** g, p_atm)
    vphi2 = np.where(inside, np.sqrt(lkep2) * R2 ** (-q) * R2, 0.0)
    prim = np.zeros((nz + 6, nphi + 6, nr + 6, 8), dtype=np.float64)
    prim[..., IRHO] = rho2[:, None, :]
    prim[..., ITAU] = p2[:, None, :]
    prim[..., IVY] = vphi2[:, None, :]
    # vector potential at cell centres, corners, then face B (model.f90:117-226)
    a_phi = np.maximum(rho2 - rho_cut, 0.0)

    def face_b(a_ph):
        a_c = np.zeros_like(a_ph)
        a_c[:-1, :-1] = 0.25 * (a_ph[:-1, :-1] + a_ph[:-1, 1:] + a_ph[1:, :-1] + a_ph[1:, 1:])
        bx = np.zeros_like(a_ph)
        bz = np.zeros_like(a_ph)
        bx[1:, :] = -(a_c[1:, :] - a_c[:-1, :]) / dz[1:, None]
        bz[:, 1:] = (xF[None, 2:] * a_c[:, 1:] - xF[None, 1:-1] * a_c[:, :-1]) / (x[None, 1:] * dx[None, 1:])
        return bx, bz

    bx, bz = face_b(a_phi)
    bxc = np.zeros_like(bx)
    bxc[:, 1:] = (xF[None, 2:] * bx[:, 1:] + xF[None, 1:-1] * bx[:, :-1]) / (xF[None, 2:] + xF[None, 1:-1])
    bzc = np.zeros_like(bz)
    bzc[1:, :] = 0.5 * (bz[1:, :] + bz[:-1, :])
    b2 = bxc ** 2 + bzc ** 2
    sel = (b2 > 0) & inside
    beta = np.min(2.0 * p2[sel] / b2[sel]) if np.any(sel) else 1.0
    b0 = math.sqrt(beta / beta_min)
    bx, bz = face_b(a_phi * b0)
    prim[..., IBX] = bx[:, None, :]
    prim[..., IBZ] = bz[:, None, :]
    rng = np.random.Generator(np.random.PCG64(seed))
    pert = 1.0 + noise * (rng.random(prim.shape[:3]) - 0.5) / 0.5
    prim[..., ITAU] = np.where(inside[:, None, :], prim[..., ITAU] * pert, prim[..., ITAU])
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    eps_floor = p_atm / rho_atm / (g - 1.0)
    spec["model"] = dict(gamma=g, floor="torus", rho_floor=rho_atm, eps_floor=eps_floor, p_floor=p_atm,
                         source="pm_cyl", r_sh=r_sh, bc="torus_cyl")
    return spec, prim, np.ascontiguousarray(eps)


def torus_cyn(nr=128, nphi=128, nz=128, faces=None, r_range=(1.5, 21.5), z_range=(-10.0, 10.0), recon="ppm",
              riemann="hlld", cfl=0.8, precision="fp64", learned=0, seed=20261203, r_sh=1.0, s_in=3.0, s_max=4.7,
              q=2.0, gamma=5.0 / 3.0, rho_max=1.0, rho_fac=1e-4, rho_cut=0.5, p_beta=350.0, noise=1e-4):
    """The reference's own cylindrical torus: GET_MODEL of
    model/torus-cyn/src/model.f90:6-316 with the values of its param.h
    (Paczynski-Wiita potential r_sh = 1, q = 2, s_in = 3, s_max = 4.7, gamma =
    5/3, atmosphere rho_fac rho_max at p = K rho^gamma, rho_cut = 0.5, minimum
    plasma beta 350, no corona) on the uniform grid of its parameter.h (r in
    [1.5, 21.5], phi in [0, 2 pi), z in [-10, 10], 128^3, boundaries
    (1,1,0,0,1,1), PPM + HLLD, CFL 0.8); ``faces`` takes a refined grid
    (CUSTOM_GRID with refine_grid).  The C5 benchmark torus (`torus_cyl`)
    is a different, Newtonian setup.

    As the reference: the field's beta normalisation averages only the
    radial face field to the cell centres (bcell(ibz) is not filled there,
    model.f90:137-145, and B_phi is zero), and the density is perturbed by
    a seeded uniform 1e-4 (model.f90:285-294)."""
    g = gamma
    spec = _base_spec(nr, nphi, nz, 3, (1, 1, 0, 0, 1, 1), r_range, (0.0, 2.0 * math.pi), z_range,
                      coordinate_flag=1, cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      learned=learned, name="torus_cyn_%dx%dx%d" % (nr, nphi, nz))
    if faces is not None:
        for key, f, n in zip(("xF", "yF", "zF"), faces, (nr, nphi, nz)):
            f = np.asarray(f, dtype=np.float64)
            if f.shape != (n + 7,):
                raise ValueError("%s needs %d faces (indices -3..n+3)" % (key, n + 7))
            spec[key] = f
    xF, zF = spec["xF"], spec["zF"]
    x, z = centers(xF), centers(zF)
    dx, dz = xF[1:] - xF[:-1], zF[1:] - zF[:-1]

    def schwarzschild(r, zz):
        return -1.0 / (np.sqrt(r ** 2 + zz ** 2) - r_sh)

    lkep2 = s_max ** (2.0 * q - 1.0) / (s_max - r_sh) ** 2
    c_const = schwarzschild(s_in, 0.0) - lkep2 * s_in ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q)
    h_max = -schwarzschild(s_max, 0.0) + lkep2 * s_max ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    k_poly = h_max * (g - 1.0) / g / rho_max ** (g - 1.0)
    if k_poly < 0.0:
        raise ValueError("The polytropic constant is negative")
    rho_a = rho_fac * rho_max
    R, Z = np.meshgrid(x, z, indexing="xy")      # (nz+6, nr+6): [l+2, j+2]
    with np.errstate(divide="ignore", invalid="ignore"):
        enth = -schwarzschild(R, Z) + lkep2 * R ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    enth = np.where(np.isfinite(enth) & (enth > 0.0), enth, 0.0)
    rho_t = (enth * (g - 1.0) / g / k_poly) ** (1.0 / (g - 1.0))
    interior = np.zeros(R.shape, dtype=bool)
    interior[3:3 + nz, 3:3 + nr] = True
    inside = (rho_t > rho_a) & (R >= s_in) & interior
    rho2 = np.where(inside, rho_t, rho_a)
    vphi2 = np.where(inside, np.sqrt(lkep2) * np.where(inside, R, 1.0) ** (-q) * R, 0.0)
    p2 = k_poly * rho2 ** g
    eps2 = k_poly * rho2 ** (g - 1.0) / (g - 1.0)
    a_phi = np.where(interior & (rho2 >= rho_cut), (rho2 - rho_cut) / rho_max, 0.0)
    xf = xF[1:]                                   # xF(j) at index j+2

    def face_b(a_ph):
        a_c = np.zeros_like(a_ph)                 # corners j, l = 1..n from cells j..j+1, l..l+1
        a_c[3:3 + nz, 3:3 + nr] = 0.25 * (a_ph[3:3 + nz, 3:3 + nr] + a_ph[3:3 + nz, 4:4 + nr]
                                           + a_ph[4:4 + nz, 3:3 + nr] + a_ph[4:4 + nz, 4:4 + nr])
        bx, bz = np.zeros_like(a_ph), np.zeros_like(a_ph)
        ll, jj = slice(2, 3 + nz), slice(2, 3 + nr)          # l, j = 0..n
        lm, jm = slice(1, 2 + nz), slice(1, 2 + nr)
        bx[ll, jj] = -(a_c[ll, jj] - a_c[lm, jj]) / dz[ll, None]
        bz[ll, jj] = (xf[None, jj] * a_c[ll, jj] - xf[None, jm] * a_c[ll, jm]) / (x[None, jj] * dx[None, jj])
        return bx, bz

    bx, bz = face_b(a_phi)
    li, ji, jim = slice(3, 3 + nz), slice(3, 3 + nr), slice(2, 2 + nr)
    bxc = np.zeros_like(bx)
    bxc[li, ji] = (xf[None, ji] * bx[li, ji] + xf[None, jim] * bx[li, jim]) / (xf[None, ji] + xf[None, jim])
    b2 = bxc ** 2
    sel = interior & (b2 > 0.0)
    beta_min = np.min(2.0 * p2[sel] / b2[sel]) if np.any(sel) else 1e30
    bx, bz = face_b(a_phi * math.sqrt(beta_min / p_beta))
    prim = np.zeros((nz + 6, nphi + 6, nr + 6, 8), dtype=np.float64)
    prim[..., IRHO] = rho2[:, None, :]
    prim[..., IVY] = vphi2[:, None, :]
    prim[..., ITAU] = p2[:, None, :]
    prim[..., IBX] = bx[:, None, :]
    prim[..., IBZ] = bz[:, None, :]
    eps = np.broadcast_to(eps2[:, None, :], prim.shape[:3]).copy()
    rho_floor = rho_max * rho_fac
    rng = np.random.Generator(np.random.PCG64(seed))
    pert = (rng.random(prim.shape[:3]) - 0.5) / 0.5 * noise
    above = (prim[..., IRHO] > rho_floor) & interior[:, None, :]
    above[:, :3, :] = False
    above[:, 3 + nphi:, :] = False
    prim[..., IRHO] = np.where(above, prim[..., IRHO] + prim[..., IRHO] * pert, prim[..., IRHO])
    spec["model"] = dict(gamma=g, floor="torus", rho_floor=rho_floor, eps_floor=k_poly * rho_floor ** (g - 1.0) / (g - 1.0),
                         p_floor=k_poly * rho_floor ** g, source="pm_cyl", r_sh=r_sh, bc="torus_cyl")
    spec["t_orbit"] = 2.0 * math.pi / (math.sqrt(lkep2) * s_max ** (-q))
    return spec, prim, np.ascontiguousarray(eps)


def torus_sph(nr=None, ntheta=None, nphi=None, faces=None, r_range=(1.5, 31.5), recon="ppm", riemann="hlld",
              cfl=0.8, precision="fp64", learned=0, seed=20261203, r_sh=1.0, s_in=3.0, s_max=4.7, q=2.0,
              gamma=5.0 / 3.0, rho_max=1.0, rho_fac=1e-4, rho_cut=0.5, p_beta=350.0, noise=1e-4, fixpole=1):
    """Torus around a pseudo-Newtonian (Paczynski-Wiita, r_sh = 1) point
    mass on a spherical (r, theta, phi) grid: GET_MODEL of
    model/torus-sph/src/model.f90:6-316 with the values of its param.h
    (q = 2, s_in = 3, s_max = 4.7, gamma = 5/3, rho_fac = 1e-4, rho_cut = 0.5,
    field scaled to the minimum plasma beta p_beta = 350, no corona).

    The grid: ``faces`` (xF, yF, zF), or nr x ntheta x nphi uniform cells
    over r_range x (0, pi) x (0, 2 pi), or by default the refined grid the
    model reads (CUSTOM_GRID, model/torus-sph/src/custom.f90:54-145), made
    by the restated generator (124 x 44 x 128 cells).  Boundaries: outflow
    in r with the torus's radial-velocity clamps, the polar axis in theta
    (with FIXPOLE), periodic in phi.  Density inside the torus
    (model.f90:84-122): H = -Phi(r) + l_K^2 s^(2-2q)/(2-2q) + C with
    Phi(r) = -1/(r - r_sh), s = r sin(theta); rho = (H (g-1)/g/K)^(1/(g-1))
    where it exceeds the atmosphere and s >= s_in, else the atmosphere
    rho_fac rho_max; p = K rho^g.  A_phi = (rho - rho_cut)/rho_max where
    rho >= rho_cut, averaged to the cell corners; the face field is its
    curl (model.f90:127-145, 209-226).  The density is perturbed by a
    seeded uniform 1e-4 (model.f90:285-294; RANDOM_NUMBER there).
    Solver defaults as the reference's solver/mhd/parameter.h ships them:
    PPM + HLLD, CFL 0.8.  The atmosphere is cold (p = K rho_atm^gamma, about
    1.7e-9 against 0.14 in the torus): WENO-Z reconstructs negative face
    pressures next to the torus within a step and the sound speed becomes
    NaN, in the reference's arithmetic as in this one, so WENO-Z needs the
    positivity fallback here.
    Returns (spec, prim, eps); cells outside 1..n hold the atmosphere until
    INITIAL_UPDATE fills the ghosts."""
    from . import grids
    g = gamma
    if faces is None and nr is None:
        nr, ntheta, nphi, r, th, ph = grids.spherical_torus_grid()
        faces = (r, th, ph)
    spec = _base_spec(nr, ntheta, nphi, 3, (1, 1, 3, 3, 0, 0), r_range, (0.0, math.pi), (0.0, 2.0 * math.pi),
                      coordinate_flag=2, cfl=cfl, recon=recon, riemann=riemann, precision=precision,
                      learned=learned, fixpole=fixpole, name="torus_sph_%dx%dx%d" % (nr, ntheta, nphi))
    if faces is not None:
        for key, f, n in zip(("xF", "yF", "zF"), faces, (nr, ntheta, nphi)):
            f = np.asarray(f, dtype=np.float64)
            if f.shape != (n + 7,):
                raise ValueError("%s needs %d faces (indices -3..n+3)" % (key, n + 7))
            spec[key] = f
    xF, yF = spec["xF"], spec["yF"]
    x, y = centers(xF), centers(yF)            # indices -2..n+3
    dx = xF[1:] - xF[:-1]
    sinf = np.sin(yF[1:])                      # indices -2..ny+3 (sinf(k) = sin(yF(k)))
    if fixpole:  # getgrid.f90:91-98, after the other metric arrays: sin 0 on the axis
        sinf[2], sinf[2 + ntheta] = 0.0, 0.0
    dcose = -(np.cos(yF[1:]) - np.cos(yF[:-1]))
    dy = yF[1:] - yF[:-1]
    dx_cb = xF[1:] ** 3 - xF[:-1] ** 3

    def schwarzschild(rr):
        return -1.0 / (rr - r_sh)

    lkep2 = s_max ** (2.0 * q - 1.0) / (s_max - r_sh) ** 2
    c_const = schwarzschild(s_in) - lkep2 * s_in ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q)
    h_max = -schwarzschild(s_max) + lkep2 * s_max ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    k_poly = h_max * (g - 1.0) / g / rho_max ** (g - 1.0)
    if k_poly < 0.0:
        raise ValueError("The polytropic constant is negative")
    rho_a = rho_fac * rho_max
    X, Y = np.meshgrid(x, y, indexing="xy")    # (ny+6, nx+6): [k+2, j+2]
    s_eq = X * np.sin(Y)
    with np.errstate(divide="ignore", invalid="ignore"):
        enth = -schwarzschild(X) + lkep2 * s_eq ** (2.0 - 2.0 * q) / (2.0 - 2.0 * q) + c_const
    enth = np.where(np.isfinite(enth) & (enth > 0.0), enth, 0.0)
    rho_t = (enth * (g - 1.0) / g / k_poly) ** (1.0 / (g - 1.0))
    inside = (rho_t > rho_a) & (s_eq >= s_in)
    interior = np.zeros_like(inside)
    interior[3:3 + ntheta, 3:3 + nr] = True      # cells 1..n, where GET_MODEL writes
    inside &= interior
    rho2 = np.where(inside, rho_t, rho_a)
    with np.errstate(divide="ignore"):
        vphi2 = np.where(inside, np.sqrt(lkep2) * np.where(inside, s_eq, 1.0) ** (-q) * s_eq, 0.0)
    p2 = k_poly * rho2 ** g
    eps2 = k_poly * rho2 ** (g - 1.0) / (g - 1.0)
    a_phi = np.where(interior & (rho2 >= rho_cut), (rho2 - rho_cut) / rho_max, 0.0)

    def face_b(a_ph):
        # corners (j, k) for j, k = 1..n from the cells j..j+1, k..k+1
        a_c = np.zeros_like(a_ph)
        a_c[3:3 + ntheta, 3:3 + nr] = 0.25 * (a_ph[3:3 + ntheta, 3:3 + nr] + a_ph[3:3 + ntheta, 4:4 + nr]
                                               + a_ph[4:4 + ntheta, 3:3 + nr] + a_ph[4:4 + ntheta, 4:4 + nr])
        bx = np.zeros_like(a_ph)
        by = np.zeros_like(a_ph)
        kk = slice(2, 3 + ntheta)                  # k = 0..ny
        jj = slice(2, 3 + nr)                      # j = 0..nx
        km, jm = slice(1, 2 + ntheta), slice(1, 2 + nr)
        xf = xF[1:]                                # xF(j) at index j+2
        bx[kk, jj] = ((sinf[kk, None] * a_c[kk, jj] - sinf[km, None] * a_c[km, jj])
                      / (xf[None, jj] * dcose[kk, None] + np.finfo(np.float64).tiny))
        by[kk, jj] = -(xf[None, jj] * a_c[kk, jj] - xf[None, jm] * a_c[kk, jm]) / (x[None, jj] * dx[None, jj])
        return bx, by

    bx, by = face_b(a_phi)
    # cell-centred field for the beta normalisation (model.f90:150-158)
    xf = xF[1:]
    bxc = np.zeros_like(bx)
    byc = np.zeros_like(by)
    ki, ji = slice(3, 3 + ntheta), slice(3, 3 + nr)
    kim, jim = slice(2, 2 + ntheta), slice(2, 2 + nr)
    bxc[ki, ji] = 1.5 * dx[None, ji] / dx_cb[None, ji] * (xf[None, ji] ** 2 * bx[ki, ji] + xf[None, jim] ** 2 * bx[ki, jim])
    byc[ki, ji] = 0.5 * dy[ki, None] / dcose[ki, None] * (sinf[ki, None] * by[ki, ji] + sinf[kim, None] * by[kim, ji])
    b2 = bxc ** 2 + byc ** 2
    sel = interior & (b2 > 0.0)
    beta_min = np.min(2.0 * p2[sel] / b2[sel]) if np.any(sel) else 1e30
    b0 = math.sqrt(beta_min / p_beta)
    bx, by = face_b(a_phi * b0)
    prim = np.zeros((nphi + 6, ntheta + 6, nr + 6, 8), dtype=np.float64)
    prim[..., IRHO] = rho2[None]
    prim[..., IVZ] = vphi2[None]
    prim[..., ITAU] = p2[None]
    prim[..., IBX] = bx[None]
    prim[..., IBY] = by[None]
    eps = np.broadcast_to(eps2[None], prim.shape[:3]).copy()
    rho_floor = rho_max * rho_fac
    rng = np.random.Generator(np.random.PCG64(seed))
    pert = (rng.random(prim.shape[:3]) - 0.5) / 0.5 * noise
    above = prim[..., IRHO] > rho_floor
    above[:, ~interior] = False
    prim[..., IRHO] = np.where(above, prim[..., IRHO] + prim[..., IRHO] * pert, prim[..., IRHO])
    spec["model"] = dict(gamma=g, floor="torus", rho_floor=rho_floor, eps_floor=k_poly * rho_floor ** (g - 1.0) / (g - 1.0),
                         p_floor=k_poly * rho_floor ** g, source="pm_sph", r_sh=r_sh, bc="torus_sph")
    spec["t_orbit"] = 2.0 * math.pi / (math.sqrt(lkep2) * s_max ** (-q))
    return spec, prim, np.ascontiguousarray(eps)


# ---------------------------------------------------------------------------
# self-gravitating star on a spherical grid: the setting of the collapsar
# model's gravity solve (model/collapsar/src/custom.f90:489-620).  The
# model itself, from the progenitor files the reference ships
# (model/collapsar/profile, read by model.f90:44-105), is collapsar_model
# below; this analytic, seeded star of the same shape (a centrally
# condensed star inside a tenuous atmosphere, rotating differentially) is
# the small, fast setting of the tests.
# ---------------------------------------------------------------------------
def star_sph(nr=96, ntheta=48, nphi=48, r_range=(2.0, 40.0), theta_range=(0.1 * math.pi, 0.9 * math.pi), rho_c=1.0,
             r_core=2.0, r_star=20.0, rho_atm=1e-6, p_atm=1e-8, asym=0.05, seed=20261203, recon="weno",
             riemann="hlld", cfl=0.4, precision="fp64"):
    """rho = rho_c / (1 + (r / r_core)^2)^1.5 inside r_star (times
    1 + asym * sin(theta) cos(phi) + 1% seeded noise), rho_atm outside;
    p = K rho^(5/3) with K = 1; v = 0, B = 0.  Returns (spec, prim, eps).

    The default theta range keeps clear of the axis.  Pole to pole, the
    rows of the cells next to the axis are strongly non-symmetric (the
    cot(theta) d/dtheta term gives the outer theta neighbour a weight
    2 / (r dtheta)^2 and the inner one about none) unless the phi coupling,
    1 / (r sin(theta) dphi)^2, dominates them; with few phi cells it does
    not, the Jacobi eigenvalues of the red-black splitting turn complex and
    over-relaxation by 1.9 diverges (48 phi cells: diverges, 1.7 converges;
    128 phi cells, the collapsar model's grid: 1.9 converges)."""
    g = 5.0 / 3.0
    full = theta_range[0] == 0.0 and theta_range[1] == math.pi
    spec = _base_spec(nr, ntheta, nphi, 3, (1, 1, 3 if full else 1, 3 if full else 1, 0, 0), r_range, theta_range,
                      (0.0, 2.0 * math.pi), coordinate_flag=2, cfl=cfl, recon=recon, riemann=riemann,
                      precision=precision, fixpole=1 if full else 0, name="star_sph_%dx%dx%d" % (nr, ntheta, nphi))
    r, th, ph = centers(spec["xF"]), centers(spec["yF"]), centers(spec["zF"])
    P3, T3, R3 = np.meshgrid(ph, th, r, indexing="ij")
    rng = np.random.Generator(np.random.PCG64(seed))
    rho = rho_c / (1.0 + (R3 / r_core) ** 2) ** 1.5
    rho = rho * (1.0 + asym * np.sin(T3) * np.cos(P3)) * (1.0 + 0.01 * (rng.random(R3.shape) - 0.5) / 0.5)
    rho = np.where(R3 < r_star, rho, rho_atm)
    prim = np.zeros((nphi + 6, ntheta + 6, nr + 6, 8), dtype=np.float64)
    prim[..., IRHO] = rho
    prim[..., ITAU] = np.where(R3 < r_star, rho ** g, p_atm)
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    spec["model"] = dict(gamma=g, floor="eps", source="none", bc="none", rho_floor=rho_atm)
    spec["rho_atm"] = rho_atm
    return spec, prim, np.ascontiguousarray(eps)


def collapsar_sph(nr=96, ntheta=48, nphi=48, m_bh=0.2, c_code=20.0, v_in=0.02, rho_c=0.01, **kw):
    """The star of star_sph set up as the collapsar model runs it: its
    floors (the atmosphere state prim_a = the outermost cell, zero velocity,
    model/collapsar/src/model.f90:238-242) and its source (self-gravity of
    the potential plus a black hole of mass m_bh; c_code = the speed of light
    in code units, r_sh = 2 m_bh / c_code^2), and an inflow of speed v_in
    that fades outward, so the hole accretes.  No magnetic field.  Returns
    (spec, prim, eps)."""
    g = 5.0 / 3.0
    spec, prim, eps = star_sph(nr, ntheta, nphi, rho_c=rho_c, **kw)
    r = centers(spec["xF"])
    rho_a = float(prim[3, 3, nr + 2, IRHO])   # prim(irho, nx, 1, 1)
    p_a = float(prim[3, 3, nr + 2, ITAU])
    prim[..., IVX] = -v_in * np.exp(-(r[None, None, :] - r[3]) / 4.0)
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    spec["boundary_flag"] = [1, 1] + list(spec["boundary_flag"][2:])
    spec["model"] = dict(gamma=g, floor="collapsar", rho_floor=rho_a, eps_floor=p_a / rho_a / (g - 1.0),
                         source="collapsar", bc="none")
    spec["rho_atm"] = rho_a
    spec["m_bh"] = m_bh
    spec["c_code"] = c_code
    spec["name"] = "collapsar_sph_%dx%dx%d" % (nr, ntheta, nphi)
    return spec, prim, np.ascontiguousarray(eps)


# ---------------------------------------------------------------------------
# the collapsar model from the progenitor files it ships
# (model/collapsar/profile/: par.dat, hydro.dat, r_grid.dat, th_grid.dat,
# phi_grid.dat)
# ---------------------------------------------------------------------------
COLLAPSAR_GRID = (156, 44, 128)   # the shipped grid files' cell counts (nx, ny, nz)


def read_collapsar_profile(directory):
    """The collapsar model's input files as GET_MODEL and CUSTOM_GRID read
    them (model/collapsar/src/model.f90:44-90, custom.f90:78-150): par.dat's
    five numbers (gamma, the black hole mass, the mass, length and time
    conversions from cgs), hydro.dat's density and pressure for cells
    -2..nx+3, and the r, theta, phi faces -3..n+3.  The cell counts follow
    from the files (the reference checks them against its compiled nx, ny,
    nz).  Returns a dict of numpy arrays."""
    import os

    from . import grids

    def numbers(name):
        with open(os.path.join(directory, name)) as f:
            return [[float(t) for t in ln.split()] for ln in f.read().splitlines() if ln.strip()]
    par = numbers("par.dat")[0]
    hydro = np.array(numbers("hydro.dat"), dtype=np.float64)
    n_r = len(numbers("r_grid.dat")) - 7
    n_th = len(numbers("th_grid.dat")) - 7
    n_ph = len(numbers("phi_grid.dat")) - 7
    if hydro.shape != (n_r + 6, 2):
        raise ValueError("inconsistent number of simulation grids: hydro.dat has %d lines, the r grid %d cells"
                         % (hydro.shape[0], n_r))
    xF, yF, zF = grids.load_grid(directory, n_r, n_th, n_ph, names=("r_grid.dat", "th_grid.dat", "phi_grid.dat"))
    return dict(par=np.array(par[:5], dtype=np.float64), rho=hydro[:, 0].copy(), p=hydro[:, 1].copy(),
                xF=xF, yF=yF, zF=zF)


def collapsar_model(profile, recon="ppm", riemann="hlld", cfl=0.8, precision="fp64", seed=20261203,
                    rotation_rule=2, w_0=10.0, b_0=1.0e10, v_crit=0.01, fixpole=1):
    """GET_MODEL of the collapsar (model/collapsar/src/model.f90:6-253) with
    the values of its param.h, from its shipped progenitor (profile = the
    dict of read_collapsar_profile, or a directory holding the files).

    Steps, in the reference's order:
      * units from par.dat: vel2code = length / time, gauss2code =
        (mass / length)^(1/2) / time; w_0 = 10 / time, b_0 = 1e10 gauss,
        v_crit = 0.01 c (model.f90:44-65, param.h);
      * rho and p of hydro.dat on every row of cells -2..nx+3, epsilon =
        p / rho / (gamma - 1) over the whole padded grid (model.f90:86-99);
      * the core radius s_core: the first cell centre j = 1..nx where the
        density rises above that of cell nx (model.f90:106-112);
      * differential rotation (rotation_rule 2, model.f90:145-167): v_phi =
        w_0 s_core^2 / (s_core^2 + s^2) s, s = x(j) sin(y(k)), where the
        density exceeds that of cell nx (rigid rotation, rule 1: v_crit / max
        x times s);
      * the field of A_phi = xF(j) sinf(k) / 2 on j, k, l = 0..n, curled onto
        the faces 0..n (model.f90:176-194) and scaled by b_0 -- a uniform
        field along the axis;
      * the density of cells 1..n above that of cell nx perturbed by a
        relative 1e-4 uniform noise, after epsilon was set (model.f90:
        220-229; the reference's RANDOM_NUMBER stream is unseeded, this one
        is PCG64(seed), drawn in the reference's loop order, l, k, j);
      * the atmosphere prim_a = (rho, 0, 0, 0, p) of cell nx and its epsilon
        (model.f90:239-242) set the floors.
    A_phi outside 0..n (read by the curl at j = 0 and k = 0) is never set by
    the reference; it is taken as zero here.
    The run configuration is not shipped for this model (the solver's
    parameter.h is set up for another one); the grid files fix a spherical
    (r, theta, phi) grid of 156 x 44 x 128 cells over the whole sphere, so
    the boundaries are outflow in r (with the model's radial-velocity clamps,
    custom.f90:160-190), the polar axis in theta (with FIXPOLE, as make.inc
    sets it) and periodic in phi; PPM + HLLD at CFL 0.8 as parameter.h ships
    them.  Self-gravity (the Poisson solve) and the black hole (mass from
    par.dat, r_sh = 2 m_bh / c^2) are the engine's collapsar source; the run
    ends at 15 s (total_time = 15 tcgs2code).  Returns (spec, prim, eps)."""
    if isinstance(profile, str):
        if profile.endswith(".npz"):  # a recorded copy of the files (tests/golden/make_collapsar_profile.py)
            with np.load(profile) as z:
                profile = {k: z[k] for k in ("par", "rho", "p", "xF", "yF", "zF")}
        else:
            profile = read_collapsar_profile(profile)
    ggas, m_bh, mass2code, length2code, t2code = (float(v) for v in profile["par"])
    xF, yF, zF = (np.asarray(profile[k], dtype=np.float64) for k in ("xF", "yF", "zF"))
    nx, ny, nz = xF.size - 7, yF.size - 7, zF.size - 7
    clight = 2.99792458e10
    vel2code = length2code / t2code
    gauss2code = (mass2code / length2code) ** 0.5 / t2code
    w0 = w_0 / t2code
    b0 = b_0 * gauss2code
    vcrit = v_crit * clight * vel2code
    spec = _base_spec(nx, ny, nz, 3, (1, 1, 3, 3, 0, 0), (float(xF[3]), float(xF[-4])), (float(yF[3]), float(yF[-4])),
                      (float(zF[3]), float(zF[-4])), coordinate_flag=2, cfl=cfl, recon=recon, riemann=riemann,
                      precision=precision, fixpole=fixpole, name="collapsar_%dx%dx%d" % (nx, ny, nz))
    spec["xF"], spec["yF"], spec["zF"] = xF.copy(), yF.copy(), zF.copy()
    x, y = centers(xF), centers(yF)            # cells -2..n+3 at index j+2
    dx = xF[1:] - xF[:-1]
    sinf = np.sin(yF)                          # faces -3..n+3 at index k+3
    if fixpole:  # getgrid.f90:91-98
        sinf[3], sinf[3 + ny] = 0.0, 0.0
    dcose = np.full(ny + 7, np.nan)
    dcose[1:] = -(np.cos(yF[1:]) - np.cos(yF[:-1]))   # k = -2..ny+3 at index k+3 (k = -1.. used)
    sine = np.sin(y)
    rho_row, p_row = np.asarray(profile["rho"], dtype=np.float64), np.asarray(profile["p"], dtype=np.float64)
    prim = np.zeros((nz + 6, ny + 6, nx + 6, 8), dtype=np.float64)
    prim[..., IRHO] = rho_row[None, None, :]
    prim[..., ITAU] = p_row[None, None, :]
    eps = prim[..., ITAU] / prim[..., IRHO] / (ggas - 1.0)
    rho_nx = rho_row[nx + 2]                  # prim(irho, nx, 1, 1)
    s_core = None
    for j in range(1, nx + 1):
        if rho_row[j - 1 + 2] <= rho_nx and rho_row[j + 2] > rho_nx:
            s_core = x[j + 2]
            break
    if s_core is None:
        raise ValueError("the progenitor's density never rises above the atmosphere's")
    inside = np.zeros((ny + 6, nx + 6), dtype=bool)
    inside[3:ny + 3, 3:nx + 3] = rho_row[None, 3:nx + 3] > rho_nx
    s_eq = x[None, :] * sine[:, None]
    if rotation_rule == 1:
        omega = vcrit / float(np.max(x))
        vphi = omega * s_eq
    else:
        sc2 = s_core * s_core
        vphi = w0 * sc2 / (sc2 + s_eq * s_eq) * s_eq
    prim[3:nz + 3, :, :, IVZ] = np.where(inside, vphi, 0.0)[None]      # l = 1..nz
    # A_phi on j, k = 0..n (zero elsewhere), the curl onto faces 0..n
    a_phi = np.zeros((ny + 6, nx + 6))
    a_phi[2:ny + 3, 2:nx + 3] = xF[None, 3:nx + 4] * sinf[3:ny + 4, None] * 0.5
    tiny = np.finfo(np.float64).tiny
    kk, jj = slice(2, ny + 3), slice(2, nx + 3)            # k, j = 0..n
    km, jm = slice(1, ny + 2), slice(1, nx + 2)            # k-1, j-1
    xf_j, xf_jm = xF[3:nx + 4], xF[2:nx + 3]               # xF(j), xF(j-1) for j = 0..nx
    sinf_k, sinf_km = sinf[3:ny + 4], sinf[2:ny + 3]       # sinf(k), sinf(k-1)
    bx = np.zeros((ny + 6, nx + 6))
    by = np.zeros((ny + 6, nx + 6))
    bx[kk, jj] = ((sinf_k[:, None] * a_phi[kk, jj] - sinf_km[:, None] * a_phi[km, jj])
                  / (xf_j[None, :] * dcose[3:ny + 4, None] + tiny))
    by[kk, jj] = -(xf_j[None, :] * a_phi[kk, jj] - xf_jm[None, :] * a_phi[kk, jm]) / (x[None, jj] * dx[None, jj])
    prim[2:nz + 3, :, :, IBX] = (bx * b0)[None]                         # l = 0..nz
    prim[2:nz + 3, :, :, IBY] = (by * b0)[None]
    # the density perturbation, in the reference's loop order
    rng = np.random.Generator(np.random.PCG64(seed))
    for l in range(1, nz + 1):
        for k in range(1, ny + 1):
            row = prim[l + 2, k + 2, 3:nx + 3, IRHO]
            sel = np.nonzero(row > rho_nx)[0]
            if sel.size:
                r = rng.random(sel.size)
                row[sel] = row[sel] * (1.0 + 1.0e-4 * (r - 0.5) / 0.5)
    p_a = p_row[nx + 2]
    eps_a = p_a / rho_nx / (ggas - 1.0)
    spec["model"] = dict(gamma=ggas, floor="collapsar", rho_floor=rho_nx, eps_floor=eps_a, source="collapsar",
                         bc="torus_sph")
    spec["rho_atm"] = rho_nx
    spec["m_bh"] = m_bh
    spec["c_code"] = clight * vel2code
    spec["t_end"] = 15.0 * t2code
    spec["s_core"] = s_core
    spec["n_pot"] = 10
    return spec, prim, np.ascontiguousarray(eps)


# ---------------------------------------------------------------------------
# named workloads
# ---------------------------------------------------------------------------
WORKLOADS = {
    "brio_wu": brio_wu,
    "blast3d": blast_3d,
    "alfven3d": alfven_3d,
    "torus_cyl": torus_cyl,
}


# ---------------------------------------------------------------------------
# smooth random state on any geometry (parity tests exercise every code path)
# ---------------------------------------------------------------------------
def smooth_state(nx, ny, nz, n_dim, coordinate_flag=0, boundary_flag=(0, 0, 0, 0, 0, 0), x_range=(0.0, 1.0),
                 y_range=(0.0, 1.0), z_range=(0.0, 1.0), seed=1, recon="weno", riemann="hlld", cfl=0.4,
                 gamma=5.0 / 3.0, precision="fp64", model=None, faces=None, **kw):
    """faces: optional (xF, yF, zF) face arrays (indices -3..n+3), e.g. the
    non-uniform grids of cumc3d_b200.grids; the ranges then follow them."""
    rng = np.random.Generator(np.random.PCG64(seed))
    spec = _base_spec(nx, ny, nz, n_dim, boundary_flag, x_range, y_range, z_range,
                      coordinate_flag=coordinate_flag, cfl=cfl, recon=recon, riemann=riemann,
                      precision=precision, model=model or dict(gamma=gamma, floor="eps"),
                      name="smooth_%dd_c%d" % (n_dim, coordinate_flag), **kw)
    if faces is not None:
        for key, f, n in zip(("xF", "yF", "zF"), faces, (nx, ny, nz)):
            f = np.asarray(f, dtype=np.float64)
            assert f.shape == (n + 7,)
            spec[key] = f
        x_range, y_range, z_range = ((float(f[3]), float(f[-4])) for f in faces)
    xf, yf, zf = spec["xF"], spec["yF"], spec["zF"]
    X = (centers(xf) - x_range[0]) / (x_range[1] - x_range[0])
    Y = (centers(yf) - y_range[0]) / (y_range[1] - y_range[0])
    Z = (centers(zf) - z_range[0]) / (z_range[1] - z_range[0])
    Zg, Yg, Xg = np.meshgrid(Z, Y, X, indexing="ij")

    def field(a):
        ph = rng.uniform(0, 2 * np.pi, 3)
        return a * (np.sin(2 * np.pi * Xg + ph[0]) * np.cos(2 * np.pi * Yg + ph[1]) + 0.5 * np.sin(2 * np.pi * Zg + ph[2]))

    prim = np.zeros((nz + 6, ny + 6, nx + 6, 8))
    prim[..., IRHO] = 1.0 + field(0.3) + 0.1 * (Xg > 0.5)
    prim[..., ITAU] = 0.6 + field(0.2) + 0.2 * (Yg > 0.4)
    prim[..., IVX] = field(0.3)
    prim[..., IVY] = field(0.3)
    prim[..., IVZ] = field(0.3)
    prim[..., IBX] = 0.5 + field(0.2)
    prim[..., IBY] = -0.3 + field(0.2)
    prim[..., IBZ] = 0.2 + field(0.2)
    g = spec["model"]["gamma"]
    eps = prim[..., ITAU] / prim[..., IRHO] / (g - 1.0)
    return spec, prim, np.ascontiguousarray(eps)
