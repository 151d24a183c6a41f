"""The FP32 candidate test of the cell-list builds, restated in numpy.

The list kernels (gems_b200/csrc/kernels.cuh, list_frame / list_r2) decide
most candidates with an FP32 squared distance and send to the exact FP64
test only those within a bound `err` of rlist^2.  The lists equal the exact
ones only if |r2_fp32 - r2| <= err for every pair near rlist.  These tests
restate the device arithmetic (float32 roundings, fused multiply-adds as one
rounding) for random boxes, cell grids and pairs near rlist, in both frames,
and check the bound.  The GPU parity tests check the lists themselves.
"""
import numpy as np
import pytest

F = np.float32


def fma32(a, b, c):
    """float32 fused multiply-add: the exact a*b + c, rounded once."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F)


def r2_fp32(x, y, z):
    return fma32(z, z, fma32(y, y, (x * x).astype(F)))


def err_bound(img, L, cell, pbc, rlist):
    sd = sd2 = dm = 0.0
    for k in range(3):
        if img:
            span = (3.0 * cell[k] if pbc[k] else L[k] + 3.0 * cell[k]) + rlist
            dk = 4.0 * 5.9604644775390625e-8 * span
        else:
            M = L[k] if pbc[k] else 4.0 * max(L[k], rlist)
            dk = 1025.0 * M * 2.3283064365386963e-10 + 2.4e-7 * rlist
        sd += dk
        sd2 += dk * dk
        dm = max(dm, dk)
    return 2.0 * (rlist + dm) * sd + sd2 + 1e-6 * rlist * rlist


def pairs_near_rlist(rng, L, pbc, rlist, n):
    """Atom i anywhere in the box, j at distance rlist * (1 +- 1e-3) along a
    random direction, wrapped into the box in periodic dims; the exact
    (float64) minimum-image vector i -> j."""
    pi = rng.random((n, 3)) * L
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    r = rlist * (1.0 + rng.uniform(-1e-3, 1e-3, n))
    pj = pi + r[:, None] * u
    keep = np.ones(n, bool)
    for k in range(3):
        if pbc[k]:
            pj[:, k] = np.mod(pj[:, k], L[k])
        else:
            keep &= (pj[:, k] >= 0) & (pj[:, k] < L[k])
    pi, pj = pi[keep], pj[keep]
    v = pj - pi
    for k in range(3):
        if pbc[k]:
            v[:, k] -= L[k] * np.round(v[:, k] / L[k])
    return pi, pj, (v * v).sum(1)


def image_frame_r2(pi, pj, L, cell, nc, pbc):
    """The image frame: coordinates relative to i's cell origin, j shifted by
    the periodic image that puts it next to i's cell (its stencil cell)."""
    ci = np.minimum((pi / cell).astype(int), nc - 1)
    cj = np.minimum((pj / cell).astype(int), nc - 1)
    o = ci * cell
    d = cj - ci
    sh = np.zeros_like(pj)
    for k in range(3):
        if pbc[k]:
            # the stencil offset in {-1, 0, 1} and its unwrapped cell
            off = np.where(d[:, k] > 1, -1, np.where(d[:, k] < -1, 1, 0))
            ux = cj[:, k] - ci[:, k] + off * nc[k]  # unwrapped relative cell in {-1, 0, 1}
            sh[:, k] = (ci[:, k] + ux - cj[:, k]) * cell[k]
    uj = (pj + sh - o).astype(F)
    ui = (pi - o).astype(F)
    x, y, z = (uj[:, 0] - ui[:, 0]), (uj[:, 1] - ui[:, 1]), (uj[:, 2] - ui[:, 2])
    return r2_fp32(x.astype(F), y.astype(F), z.astype(F))


def integer_frame_r2(pi, pj, L, pbc, rlist):
    comps = []
    for k in range(3):
        M = L[k] if pbc[k] else 4.0 * max(L[k], rlist)
        ls = 4294967296.0 / M
        unit = F(M * 2.384185791015625e-07)
        a = (np.rint(pi[:, k] * ls).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
        b = (np.rint(pj[:, k] * ls).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
        dv = (b.astype(np.int64) - a.astype(np.int64)) & 0xFFFFFFFF
        dv = dv.astype(np.uint32).view(np.int32) >> 10
        comps.append((dv.astype(F) * unit).astype(F))
    return r2_fp32(*comps)


@pytest.mark.parametrize("seed", range(6))
def test_image_frame_within_bound(seed):
    rng = np.random.default_rng(seed)
    rlist = rng.uniform(3.0, 8.0)
    nc = rng.integers(3, 40, 3)
    L = nc * rlist * rng.uniform(1.01, 1.3, 3)  # cells a little wider than rlist
    cell = L / nc
    pbc = [bool(b) for b in rng.integers(0, 2, 3)]
    pbc[0] = True
    pi, pj, r2 = pairs_near_rlist(rng, L, pbc, rlist, 200000)
    r2f = image_frame_r2(pi, pj, L, cell, nc, pbc)
    err = err_bound(True, L, cell, pbc, rlist)
    assert np.abs(r2f.astype(np.float64) - r2).max() <= err


@pytest.mark.parametrize("seed", range(6))
def test_integer_frame_within_bound(seed):
    rng = np.random.default_rng(100 + seed)
    rlist = rng.uniform(3.0, 8.0)
    L = rng.uniform(1.2, 400.0, 3) * np.array([1.0, 1.0, 1.0])
    L[0] = max(L[0], 4 * rlist)
    pbc = [True, bool(rng.integers(0, 2)), bool(rng.integers(0, 2))]
    pi, pj, r2 = pairs_near_rlist(rng, L, pbc, rlist, 200000)
    r2f = integer_frame_r2(pi, pj, L, pbc, rlist)
    err = err_bound(False, L, L / np.maximum(1, (L / rlist).astype(int)), pbc, rlist)
    assert np.abs(r2f.astype(np.float64) - r2).max() <= err
