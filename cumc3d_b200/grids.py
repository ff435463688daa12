"""Non-uniform grids: the face-coordinate files the torus models read, and
the generators that write them.

* ``read_faces`` / ``load_grid`` follow CUSTOM_GRID of the torus models
  (model/torus-cyn/src/custom.f90:54-141, the same in torus-sph): one face
  coordinate per line, indices -3..n+3, so a file for n cells has n + 7
  lines; any other count is an error, with the reference's message.
* ``spherical_torus_grid`` restates model/torus-sph/grid/grid.py: radial
  faces in geometric progression from xl to xr with three linear ghost faces
  below (0, xl/3, 2xl/3), theta faces stretched geometrically from the
  equator (spacing dphi at the equator, ratio from a bisection) and mirrored
  through the poles, uniform phi; the cell counts nx, ny come from
  bisections on the aspect ratios ratio_x = dr/(r dphi) and ratio_y = the
  cell aspect at the pole.
* ``cylindrical_torus_grid`` restates model/torus-cyn/grid/grid.py: the same
  radial faces, z faces with the radial spacings mirrored about z = 0,
  uniform phi.

The arrays feed ``spec["xF"]`` etc. of the models (face indices -3..n+3);
the engine builds its metric and reconstruction weights from them
(getgrid.f90, the WENO/PPM/TVD weight routines), so non-uniform spacing
needs no other change.
"""
import math

import numpy as np


def read_faces(path, n, axis="r"):
    """Face coordinates -3..n+3 from a CUSTOM_GRID file (one value per line)."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    if len(lines) != n + 7:
        raise ValueError("number of %s-grid faces from files %d, in the program %d: "
                         "inconsistent number of %s-grid faces" % (axis, len(lines) - 7, n, axis))
    return np.array([float(ln.split()[0]) for ln in lines], dtype=np.float64)


def write_faces(path, faces):
    """One face per line, shortest round-trip decimal (as the generators write)."""
    with open(path, "w") as f:
        for v in np.asarray(faces, dtype=np.float64):
            f.write(repr(float(v)) + "\n")


def load_grid(directory, nx, ny, nz, names=("r_grid.dat", "phi_grid.dat", "z_grid.dat")):
    """(xF, yF, zF) of a model's grid directory; names in axis order (the
    cylindrical torus reads r, phi, z; the spherical one r, theta, phi)."""
    import os
    return tuple(read_faces(os.path.join(directory, nm), n, ax)
                 for nm, n, ax in zip(names, (nx, ny, nz), ("x", "y", "z")))


def _bisect(f, lo, hi):
    """The generators' bisection: 100 halvings keeping the sign change."""
    f_lo, f_hi = f(lo), f(hi)
    c = lo
    for _ in range(100):
        c = 0.5 * (lo + hi)
        f_c = f(c)
        if f_c * f_lo > 0:
            lo = c
        elif f_c * f_hi > 0:
            hi = c
    return c


def _radial_faces(xl, xr, nx):
    deps = np.log(xr / xl) / nx
    r = np.zeros(nx + 7)
    dr = xl / 3
    for i in range(0, 4):
        r[i] = i * dr
    for i in range(4, nx + 7):
        r[i] = r[i - 1] * np.exp(deps)
    return r


def _count(log_ratio, xl, xr, hi):
    def g(nx):
        return nx * log_ratio - np.log(xr / xl)
    n = int(_bisect(g, 1, hi))
    return n + 1 if n % 2 else n


def spherical_torus_grid(xl=1.5, xr=31.5, ratio_x=0.5, ratio_y=0.05, nz=128):
    """(nx, ny, nz, r_faces, theta_faces, phi_faces) of the spherical torus."""
    alpha_y = np.arcsin(ratio_y) * nz / math.pi

    def strech_y(ny):
        n_grid = float(ny / 2)
        r_ratio = alpha_y ** (1 / (n_grid - 1))
        return (r_ratio ** n_grid - 1) / (r_ratio - 1) - float(nz / 4)
    ny = int(_bisect(strech_y, 1, 256))
    if ny % 2:
        ny += 1
    nx = _count(np.log((nz + ratio_x * math.pi) / (nz - ratio_x * math.pi)), xl, xr, 256)
    r = _radial_faces(xl, xr, nx)

    def strech(r_in):
        n_grid = float(ny / 2)
        return (r_in ** n_grid - 1) / (r_in - 1) - float(nz / 4)
    ratio = _bisect(strech, 1.01, 3.01)
    th = np.zeros(ny + 7)
    dphi = 2 * math.pi / nz
    h = 3 + ny // 2
    th[h] = math.pi / 2
    for i in range(h + 1, 3 + ny + 1):
        th[i] = th[i - 1] + dphi * ratio ** (i - h - 1)
    th[3 + ny] = math.pi
    for i in range(3 + ny + 1, 3 + ny + 4):
        th[i] = th[i - 1] + (th[2 * (3 + ny) - i + 1] - th[2 * (3 + ny) - i])
    for i in range(h - 1, 2, -1):
        th[i] = math.pi - th[6 + ny - i]
    for i in range(2, -1, -1):
        th[i] = -th[6 - i]
    ph = np.array([dphi * (i - 3) for i in range(nz + 7)])
    # with too few phi cells the equatorial spacing dphi is so wide that no
    # stretching ratio in the bisection's bracket (1.01, 3.01) fits ny/2 cells
    # into pi/2; the faces would come out non-monotone (nz >= 96 works at the
    # default ratios)
    if not (np.all(np.diff(th) > 0) and th[3] == 0.0 and th[3 + ny] == math.pi):
        raise ValueError("no theta stretching for nz=%d, ratio_y=%g: the faces are not monotone" % (nz, ratio_y))
    return nx, ny, nz, r, th, ph


def cylindrical_torus_grid(xl=1.5, xr=21.5, ratio_x=0.4, nphi=128):
    """(nr, nphi, nz, r_faces, phi_faces, z_faces) of the cylindrical torus."""
    nx = _count(np.log((nphi + ratio_x * math.pi) / (nphi - ratio_x * math.pi)), xl, xr, 1024)
    nz = nx
    r = _radial_faces(xl, xr, nx)
    dr = np.array([r[i + 1] - r[i] for i in range(nx + 6)])
    z = np.zeros(nz + 7)
    h = 3 + nz // 2
    for i in range(h + 1, 3 + nz + 4):
        z[i] = z[h] + np.sum(dr[3:3 + (i - h)])
    for i in range(h - 1, -1, -1):
        z[i] = -z[(h - 1 - i) + h + 1]
    dphi = 2 * math.pi / nphi
    ph = np.array([dphi * (i - 3) for i in range(nphi + 7)])
    return nx, nphi, nz, r, ph, z
