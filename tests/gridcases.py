"""Grid arrays for the general-grid tests, shaped (jpj+2, jpi+2) over the
reference's (0:jpi+1, 0:jpj+1) index range (ji fastest).

default_grid restates what original/nemolite2d.f90's `grid` (CASE 1,
:184-233) and the depth loops (:238-254) fill: every metric only over its
own point set, zero elsewhere.  random_grid builds a general one: open water
on parts of all four borders (so the Flather conditions on u and v both act),
land islands, scale factors (within 15% of dx, dy) and latitudes that vary
smoothly per point, and one smooth bathymetry between 25 and 75 m.
"""
import numpy as np

NAMES = ("e1t", "e2t", "e1u", "e2u", "e1v", "e2v", "gphiu", "gphiv", "ht", "hu", "hv")


def _ranges(jpi, jpj):
    t = (slice(1, jpj + 1), slice(1, jpi + 1))   # (1:jpi, 1:jpj)
    u = (slice(1, jpj + 1), slice(0, jpi + 1))   # (0:jpi, 1:jpj)
    v = (slice(0, jpj + 1), slice(1, jpi + 1))   # (1:jpi, 0:jpj)
    return t, u, v


def default_grid(jpi, jpj, dx=1000.0, dy=1000.0, lat=50.0, dep=100.0):
    shape = (jpj + 2, jpi + 2)
    pt = np.ones(shape, np.int32)
    pt[:, 0] = 0
    pt[:, jpi + 1] = 0
    pt[jpj + 1, :] = 0
    pt[0, 1:jpi + 1] = -1
    t, u, v = _ranges(jpi, jpj)
    g = {n: np.zeros(shape) for n in NAMES}
    g["e1t"][t], g["e2t"][t] = dx, dy
    g["e1u"][u], g["e2u"][u], g["gphiu"][u] = dx, dy, lat
    g["e1v"][v], g["e2v"][v], g["gphiv"][v] = dx, dy, lat
    g["ht"][t], g["hu"][u], g["hv"][v] = dep, dep, dep
    return pt, g


def random_grid(seed, jpi, jpj, dx=1000.0, dy=1000.0):
    rng = np.random.default_rng(seed)
    shape = (jpj + 2, jpi + 2)
    pt = np.ones(shape, np.int32)
    pt[:, 0] = 0
    pt[:, jpi + 1] = 0
    pt[0, :] = 0
    pt[jpj + 1, :] = 0

    def span(n):
        a = int(rng.integers(1, n // 2))
        return a, int(rng.integers(a + 2, n))

    a, b = span(jpi)
    pt[0, a:b] = -1            # south
    a, b = span(jpi)
    pt[jpj + 1, a:b] = -1      # north
    a, b = span(jpj)
    pt[a:b, 0] = -1            # west
    a, b = span(jpj)
    pt[a:b, jpi + 1] = -1      # east
    for _ in range(4):         # islands, clear of the border ring
        y0 = int(rng.integers(3, jpj - 4))
        x0 = int(rng.integers(3, jpi - 4))
        pt[y0:y0 + int(rng.integers(1, 4)), x0:x0 + int(rng.integers(1, 4))] = 0
    t, u, v = _ranges(jpi, jpj)
    # smooth fields with random phases, evaluated where each point set sits
    # (u half a cell east of T, v half a cell north); white noise in the
    # metrics or depths makes the reference scheme unstable within a few
    # hundred steps
    jj, ji = np.mgrid[0:jpj + 2, 0:jpi + 2].astype(np.float64)
    pos = {"t": (ji, jj), "u": (ji + 0.5, jj), "v": (ji, jj + 0.5)}

    def smooth(at, amp):
        kx, ky = rng.uniform(0.5, 2.0, 2)
        p1, p2 = rng.uniform(0.0, 2.0 * np.pi, 2)
        x, y = pos[at]
        return amp * np.sin(2 * np.pi * kx * x / jpi + p1) * np.cos(2 * np.pi * ky * y / jpj + p2)

    g = {n: np.zeros(shape) for n in NAMES}
    for name, rg, base, at in (("e1t", t, dx, "t"), ("e2t", t, dy, "t"), ("e1u", u, dx, "u"),
                               ("e2u", u, dy, "u"), ("e1v", v, dx, "v"), ("e2v", v, dy, "v")):
        g[name][rg] = (base * (1.0 + smooth(at, 0.15)))[rg]
    g["gphiu"][u] = (45.0 + smooth("u", 15.0))[u]
    g["gphiv"][v] = (45.0 + smooth("v", 15.0))[v]
    depth = [rng.uniform(0.5, 2.0, 2), rng.uniform(0.0, 2.0 * np.pi, 2)]
    for name, rg, at in (("ht", t, "t"), ("hu", u, "u"), ("hv", v, "v")):
        x, y = pos[at]  # one bathymetry seen at the three point sets
        h = 50.0 + 25.0 * np.sin(2 * np.pi * depth[0][0] * x / jpi + depth[1][0]) * \
            np.cos(2 * np.pi * depth[0][1] * y / jpj + depth[1][1])
        g[name][rg] = h[rg]
    return pt, g
