"""Seeded synthetic phantoms for the projector workloads.

Random-ellipse phantoms stand in for the FORBILD head of the reference
(python/FORBILD.py:19-181 holds that table; it is not reproduced here): the
method follows FORBILD.py:183-210 (point-sampled rasterisation) and
FORBILD.py:213-353 (closed-form chord lengths through ellipses), with
ellipse parameters drawn from a seeded generator:

* centres   U[-0.7, 0.7] * R
* semi-axes U[0.05, 0.5] * R
* angles    U[0, pi)
* densities U[-0.5, 1]

R is half the field of view.  Basis coefficients are point samples at the
pixel (or lattice-site) centres.
"""
from __future__ import annotations

import numpy as np


def random_ellipses(seed: int, n: int = 10, radius: float = 1.0) -> np.ndarray:
    """Return an (n, 6) array of (cx, cy, a, b, phi, rho) in physical units."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.7, 0.7, size=(n, 2)) * radius
    ax = rng.uniform(0.05, 0.5, size=(n, 2)) * radius
    phi = rng.uniform(0.0, np.pi, size=n)
    rho = rng.uniform(-0.5, 1.0, size=n)
    return np.column_stack([c, ax, phi, rho])


def sample_ellipses(ell: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Sum of ellipse indicator functions times density at points (x, y)."""
    out = np.zeros(np.broadcast(x, y).shape, dtype=np.float64)
    for cx, cy, a, b, phi, rho in ell:
        c, s = np.cos(phi), np.sin(phi)
        xr = (x - cx) * c + (y - cy) * s
        yr = -(x - cx) * s + (y - cy) * c
        out += rho * ((xr / a) ** 2 + (yr / b) ** 2 <= 1.0)
    return out


def pixel_centres(nx: int, ny: int, dx: float, dy: float):
    """Pixel-centre coordinates ((i - (n-1)/2) * d), layers/A_B1.cu:96-98.

    Returned as arrays indexed [ix, iy], i.e. the host layout x[ix*ny + iy]
    used by the reference C entry points (layers/A_B1.cu:621-623).
    """
    xs = (np.arange(nx) - 0.5 * (nx - 1)) * dx
    ys = (np.arange(ny) - 0.5 * (ny - 1)) * dy
    return np.meshgrid(xs, ys, indexing="ij")


def ellipse_phantom(nx: int, ny: int, dx: float, dy: float, seed: int = 0, n: int = 10) -> np.ndarray:
    """Seeded 2D ellipse phantom, float64 array of shape (nx, ny)."""
    radius = 0.5 * min(nx * dx, ny * dy)
    ell = random_ellipses(seed, n, radius)
    x, y = pixel_centres(nx, ny, dx, dy)
    return sample_ellipses(ell, x, y)


def ellipse_phantom_average(nx: int, ny: int, dx: float, dy: float, seed: int = 0, n: int = 10,
                            sub: int = 8) -> np.ndarray:
    """The same phantom averaged over each pixel (FP64, sub x sub samples per
    pixel at the centres of its sub-cells): the image a perfect reconstruction
    in pixels would hold, the ground truth of the reconstruction experiments."""
    radius = 0.5 * min(nx * dx, ny * dy)
    ell = random_ellipses(seed, n, radius)
    x, y = pixel_centres(nx, ny, dx, dy)
    off = (np.arange(sub) + 0.5) / sub - 0.5
    out = np.zeros((nx, ny), dtype=np.float64)
    for ox in off:
        for oy in off:
            out += sample_ellipses(ell, x + ox * dx, y + oy * dy)
    return out / (sub * sub)


def ellipse_chords(ell: np.ndarray, px, py, qx, qy) -> np.ndarray:
    """Line integrals of the ellipse phantom along the lines through P and Q.

    Closed-form chord lengths (the method of FORBILD.py:213-353): for each
    ellipse, the line is mapped to the unit-circle frame and the chord length
    2*sqrt(1 - d^2) is scaled back by the direction's stretch.
    """
    px, py, qx, qy = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (px, py, qx, qy)))
    dirx, diry = qx - px, qy - py
    norm = np.hypot(dirx, diry)
    dirx, diry = dirx / norm, diry / norm
    total = np.zeros(px.shape, dtype=np.float64)
    for cx, cy, a, b, phi, rho in ell:
        c, s = np.cos(phi), np.sin(phi)
        ox = ((px - cx) * c + (py - cy) * s) / a
        oy = (-(px - cx) * s + (py - cy) * c) / b
        vx = (dirx * c + diry * s) / a
        vy = (-dirx * s + diry * c) / b
        vv = vx * vx + vy * vy
        t0 = -(ox * vx + oy * vy) / vv
        d2 = (ox + t0 * vx) ** 2 + (oy + t0 * vy) ** 2
        half = np.sqrt(np.maximum(0.0, 1.0 - d2) / vv)
        total += rho * 2.0 * half
    return total


def ellipsoid_phantom(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, seed: int = 0,
                      n: int = 10) -> np.ndarray:
    """Seeded 3D phantom of random ellipsoids (rotation about z), shape (nz, ny, nx).

    Same distributions as the 2D family; the third semi-axis and the z centre
    are drawn from the same ranges.  Layout [z][y][x] as layers/A_B1_3D.cu:716.
    """
    radius = 0.5 * min(nx * dx, ny * dy, nz * dz)
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.7, 0.7, size=(n, 3)) * radius
    ax = rng.uniform(0.05, 0.5, size=(n, 3)) * radius
    phi = rng.uniform(0.0, np.pi, size=n)
    rho = rng.uniform(-0.5, 1.0, size=n)
    zs = (np.arange(nz) - 0.5 * (nz - 1)) * dz
    ys = (np.arange(ny) - 0.5 * (ny - 1)) * dy
    xs = (np.arange(nx) - 0.5 * (nx - 1)) * dx
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    for k in range(n):
        cs, sn = np.cos(phi[k]), np.sin(phi[k])
        xr = (x - c[k, 0]) * cs + (y - c[k, 1]) * sn
        yr = -(x - c[k, 0]) * sn + (y - c[k, 1]) * cs
        zr = z - c[k, 2]
        out += rho[k] * ((xr / ax[k, 0]) ** 2 + (yr / ax[k, 1]) ** 2 + (zr / ax[k, 2]) ** 2 <= 1.0)
    return out


def hex_sites(nl: int, nc: int, dt: float, row_pitch: float):
    """Site centres of the hexagonal lattice of layers/A_H0.cu:174-183 (H0:
    row_pitch = 1.5 dt; Hl: 0.5 dt, layers/A_Hl.cu:184-193), as arrays indexed
    [ic, il] (host layout x[ic*nl + il]); odd rows have nc-1 sites, the last
    column of odd rows is not a site (mask False)."""
    ic, il = np.meshgrid(np.arange(nc), np.arange(nl), indexing="ij")
    dx = dt * np.sqrt(3.0)
    shift = np.where(il % 2 == 1, 0.5 * (nc - 2), 0.5 * (nc - 1))
    x = (ic - shift) * dx
    y = (il - 0.5 * (nl - 1)) * row_pitch
    mask = ~((il % 2 == 1) & (ic == nc - 1))
    return x, y, mask


def hex_phantom(nl: int, nc: int, dt: float, row_pitch: float, seed: int = 0, n: int = 10) -> np.ndarray:
    """Seeded ellipse phantom sampled at the hexagonal sites, float64 (nc, nl)."""
    x, y, mask = hex_sites(nl, nc, dt, row_pitch)
    radius = 0.5 * min(np.ptp(x[mask]), np.ptp(y[mask]))
    out = sample_ellipses(random_ellipses(seed, n, radius), x, y)
    out[~mask] = 0.0
    return out
