"""Geometries used by the parity tests (sizes of the benchmark configurations
and small cases the CPU oracle finishes in seconds)."""
import numpy as np

LSD, LSO = 1085.6, 595.0


def fan_case(name):
    """(nx, ny, nu, dx, dy, du, lsd, lso, angles) of a named fan-beam case."""
    if name == "fan512":  # 512^2 at 0.5 mm, 720 views over 2pi, 736 bins at 1 mm
        return 512, 512, 736, 0.5, 0.5, 1.0, LSD, LSO, 2 * np.pi * np.arange(720) / 720
    if name == "small":   # 128^2 at 2 mm, 180 views, 185 bins at 1 mm
        return 128, 128, 185, 2.0, 2.0, 1.0, LSD, LSO, 2 * np.pi * np.arange(180) / 180
    if name == "rect":    # nx != ny, anisotropic pixels, odd sizes
        return 97, 64, 151, 1.5, 2.0, 1.3, LSD, LSO, 2 * np.pi * np.arange(37) / 37 + 0.1
    if name == "tiny":    # one view, few bins
        return 16, 16, 24, 1.0, 1.0, 1.0, 40.0, 20.0, np.array([0.3])
    if name == "snap":    # views exactly at odd multiples of 45 degrees (the reference's singular path)
        return 64, 64, 96, 1.0, 1.0, 1.0, 200.0, 100.0, np.array([np.pi / 4, 3 * np.pi / 4, 5 * np.pi / 4, 7 * np.pi / 4, 0.0, np.pi / 2])
    if name == "wide":    # detector narrower than the object: truncated projections
        return 96, 96, 40, 1.0, 1.0, 1.0, 300.0, 150.0, 2 * np.pi * np.arange(24) / 24
    raise KeyError(name)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def hex_case(name):
    """(nl, nc, nu, dt, du, lsd, lso, angles) of a hexagonal-lattice case."""
    if name == "small":      # 64 rows of 40 sites at dt = 2 mm
        return 64, 40, 300, 2.0, 1.5, LSD, LSO, 2 * np.pi * np.arange(90) / 90
    if name == "tall":       # Hl-like row pitch: more rows
        return 128, 40, 300, 2.0, 1.5, LSD, LSO, 2 * np.pi * np.arange(90) / 90
    if name == "h0_2e18":    # ~2^18 sites over 512 mm, 360 views x 736 bins
        return 550, 477, 736, 0.62, 1.0, LSD, LSO, 2 * np.pi * np.arange(360) / 360
    if name == "hl_2e18":
        return 953, 275, 736, 1.075, 1.0, LSD, LSO, 2 * np.pi * np.arange(360) / 360
    raise KeyError(name)


def cone_case(name):
    """(nx, ny, nz, nu, nv, dx, dy, dz, du, dv, lsd, lso, angles) of a cone-beam case."""
    if name == "small":   # 32^3 at 2 mm, 24 views, 48 x 40 detector at 3 mm
        return 32, 32, 32, 48, 40, 2.0, 2.0, 2.0, 3.0, 3.0, LSD, LSO, 2 * np.pi * np.arange(24) / 24
    if name == "rect":    # anisotropic, non-cubic, odd sizes, a snapped 45-degree view
        return 27, 20, 45, 40, 52, 2.0, 2.5, 1.5, 3.0, 2.0, LSD, LSO, np.array([0.3, np.pi / 4, 2.0, 3 * np.pi / 4 + 0.01])
    if name == "tiny":    # 16^3 at 2 mm, 8 views, 24 x 20 detector at 3 mm (golden vectors)
        return 16, 16, 16, 24, 20, 2.0, 2.0, 2.0, 3.0, 3.0, LSD, LSO, 2 * np.pi * np.arange(8) / 8
    if name == "tallz":   # 80 slices (two 64-slice chunks) past both detector edges, narrow detector
        return 16, 8, 80, 16, 20, 2.0, 2.0, 2.0, 3.0, 3.0, LSD, LSO, np.array([0.1, 1.3, np.pi / 4, 2.9, 4.4, 5.7])
    if name == "cone256": # 256^3 at 1 mm, 360 views over 2 pi, 384 x 384 at 1.5 mm
        return 256, 256, 256, 384, 384, 1.0, 1.0, 1.0, 1.5, 1.5, LSD, LSO, 2 * np.pi * np.arange(360) / 360
    raise KeyError(name)
