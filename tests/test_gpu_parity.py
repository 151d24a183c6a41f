"""CUDA path (through the C ABI) against the FP64 oracle and the golden files.

Tolerances:
  * neighbour lists: identical, entry by entry (bit-exact integer sets and
    the reference's order);
  * plain FP64 kernels: forces to 1e-10 relative RMS, energies to 1e-9 eV
    per atom (summation order and exp/sqrt implementations differ);
  * mixed kernels (FP32 pair math, FP64 accumulation): forces <= 1e-5
    relative RMS, energies <= 1e-6 eV per atom;
  * trajectories against golden files: the rule of examples/test.sh.
"""
import numpy as np
import pytest

import decks
from oracle import oracle as O

gems = pytest.importorskip("gems_b200")
pytestmark = pytest.mark.gpu

RMS_FP64 = 1e-10
E_FP64 = 1e-9        # eV per atom
RMS_MIXED = 1e-5
E_MIXED = 1e-6       # eV per atom


@pytest.fixture(scope="module")
def ctx():
    c = gems.Context()
    yield c
    c.close()


def relrms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def both(pos, mass, ctx, types=None, ntypes=1, setup=None):
    o = O.System(pos, mass, types, ntypes)
    g = gems.System(pos, mass, types, ntypes, ctx=ctx)
    for s in (o, g):
        setup(s)
    return o, g


def compare_lists(o, g, drop_self=False):
    no, lo = o.neighbour_list()
    ng, lg = g.neighbour_list()
    if drop_self:  # leave out the reference's self entries (test_list_cells_thin_slab)
        rows = [[j for j in lo[: no[i], i] if j != i] for i in range(len(no))]
        no = np.array([len(r) for r in rows])
        lo = np.zeros_like(lo)
        for i, r in enumerate(rows):
            lo[: len(r), i] = r
    np.testing.assert_array_equal(ng, no)
    m = int(no.max()) if len(no) else 0
    for k in range(m):
        mask = no > k
        np.testing.assert_array_equal(lg[k][mask], lo[k][mask])


# ------------------------------------------------------------------ lists
def smatb_bulk_setup(s, half=False):
    d = decks.bulk_deck()
    s.set_box(d["box"], d["pbc"])
    s.set_smatb(*d["smatb"])
    s.set_half(half)


@pytest.mark.parametrize("half", [False, True])
def test_list_cells_open_box(ctx, half):
    """bulk.gms geometry: boxed, no PBC, 8^3 linked cells."""
    d = decks.bulk_deck()
    rng = np.random.default_rng(7)
    pos = d["pos"] + rng.normal(0, 0.05, d["pos"].shape)
    o, g = both(pos, d["mass"], ctx, setup=lambda s: smatb_bulk_setup(s, half))
    o.update()
    g.update()
    assert o.uses_cells()[0]
    compare_lists(o, g)


@pytest.mark.parametrize("half", [False, True])
def test_list_cells_pbc_32k(ctx, half):
    from gems_b200 import workloads as W
    w = W.smatb_bulk()

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        s.set_smatb(*w["smatb"])
        s.set_half(half)

    o, g = both(w["pos"], w["mass"], ctx, setup=setup)
    o.update()
    g.update()
    assert o.uses_cells() == (True, (13, 13, 13))
    compare_lists(o, g)


@pytest.mark.parametrize("half", [False, True])
def test_list_cells_small_cells(ctx, half):
    """Cells of about three atoms (a thermal Tersoff diamond, 4.1 A cells)
    go to the warp-per-cell list kernel: the lists equal the oracle's, entry
    by entry, full and half."""
    from gems_b200 import workloads as W
    rng = np.random.default_rng(31)
    L = 10 * 5.431
    pos = np.mod(W.diamond(10, 5.431) + rng.normal(0, 0.1, (8000, 3)), L)

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
        s.set_half(half)

    o, g = both(pos, W.MASS["Si"], ctx, setup=setup)
    o.update()
    g.update()
    assert o.uses_cells() == (True, (13, 13, 13))
    compare_lists(o, g)
    g.destroy()


def test_list_cells_batch_rebuild(ctx):
    """A batch of periodic cell-list systems rebuilt together (the force
    rebuild of a kernel timing call, then md steps that rebuild each system
    at its own time): every system's list equals the oracle's, entry by
    entry, at its own positions."""
    from gems_b200 import workloads as W
    ss, os_ = [], []
    for k in range(4):
        w = W.smatb_bulk(seed=40 + k, ncell=8)

        def setup(s, w=w):
            s.set_box(w["L"], (True, True, True))
            s.set_smatb(*w["smatb"])
        o, g = both(w["pos"], w["mass"], ctx, setup=setup)
        g.set_ermak(0.002, 1.0, 900.0 + 100 * k, seed=7 + k)
        g.interact()
        ss.append(g)
        os_.append(o)
    ctx.batch_time_kernels(ss, 1)          # forces a rebuild of all four
    for o, g in zip(os_, ss):
        o.set_pos(g.pos)
        o.update()
        compare_lists(o, g)
    n0 = [g.nupd for g in ss]
    ctx.batch_md_steps(ss, 400)            # hot: each rebuilds on its own skin test
    assert all(g.nupd > n for g, n in zip(ss, n0))
    ctx.batch_time_kernels(ss, 1)
    for o, g in zip(os_, ss):
        o.set_pos(g.pos)
        o.update()
        compare_lists(o, g)
    for g in ss:
        g.destroy()


@pytest.mark.parametrize("half", [False, True])
def test_list_n2_mic(ctx, half):
    """readxyz.gms geometry: rc+skin > box/2, O(N^2) list with minimum image."""
    d = decks.xyz_deck()

    def setup(s):
        s.set_box(d["box"], (True, True, True))
        s.set_lj(*d["lj"])
        s.set_half(half)

    o, g = both(d["frames"][0], 12.0, ctx, setup=setup)
    o.update()
    g.update()
    assert not o.uses_cells()[0]
    compare_lists(o, g)


def test_list_boundary_ties(ctx):
    """A pair exactly at rlist: kept by the O(N^2) list (<=), dropped by the
    linked cells (<), as in the reference."""
    rl = 5.0 + 1.0
    pos = np.array([[1.0, 1.0, 1.0], [1.0 + rl, 1.0, 1.0], [3.0, 4.0, 1.0]])
    for boxed in (False, True):
        def setup(s):
            if boxed:
                s.set_box((40.0, 40.0, 40.0), (False, False, False))
            s.set_smatb(0.2061, 1.79, 10.229, 4.036, 2.884, 4.4, 5.0)
        o, g = both(pos, 196.97, ctx, setup=setup)
        o.update()
        g.update()
        assert o.uses_cells()[0] == boxed
        compare_lists(o, g)


@pytest.mark.parametrize("natoms", [600, 300, 90])
@pytest.mark.parametrize("pbc", [(True, True, True), (True, True, False)])
@pytest.mark.parametrize("half", [False, True])
def test_list_cells_thin_slab(ctx, pbc, half, natoms):
    """A slab one cell thick (6 x 5 x 1 cells): the stencil visits the one
    z-cell three times, so a periodic slab lists a neighbour once per visit,
    as the reference does; the lists equal the oracle's, entry by entry.
    One deliberate difference: the reference's half-list loop
    (linkedcell_selfhalf, src/Neighbour.F90:1117-1149) has no i /= j test, so
    in a periodic slab one cell thick a half-stencil cell that wraps onto the
    atom's own cell lists the atom as its own neighbour (at distance 0, which
    the force loops would then evaluate).  The GPU lists never hold an atom
    itself; the half-list comparison leaves those entries out.  (The stencil
    wraps cells in every dim, periodic or not, as cell_pbc does, so the
    slab's open z takes the same path.)  600, 300 and 90 atoms (20, 10 and 3
    per cell) reach the three list kernels (a CTA per cell, a warp per cell
    with a 512- and a 128-candidate tile) in the integer frame that a
    periodic dimension of fewer than three cells needs."""
    rng = np.random.default_rng(5)
    L = (40.0, 33.0, 7.5)
    pos = rng.random((natoms, 3)) * np.array(L)

    def setup(s):
        s.set_box(L, pbc)
        s.set_smatb(0.2061, 1.79, 10.229, 4.036, 2.884, 4.4, 5.0)
        s.set_half(half)

    o, g = both(pos, 196.97, ctx, setup=setup)
    o.update()
    g.update()
    assert o.uses_cells() == (True, (6, 5, 1))
    compare_lists(o, g, drop_self=half)
    g.destroy()


def test_list_cells_pairs_at_rlist_large_box(ctx):
    """Pairs 1e-12 relative inside and outside rlist, across the periodic
    faces of a 400 A box in every direction: the cell lists keep exactly the
    inside ones, as the oracle does."""
    rl = 5.0 + 1.0
    L = 400.0
    rng = np.random.default_rng(17)
    pts = []
    for k in range(40):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        a = rng.random(3) * L
        d = k % 3  # near a face in dim d
        a[d] = rng.random() * 3.0 + (0.1 if rng.random() < 0.5 else L - 3.1)
        r = rl * (1.0 - 1e-12 if k % 2 == 0 else 1.0 + 1e-12)
        pts += [a, np.mod(a + r * u, L)]
    pos = np.array(pts)

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_smatb(0.2061, 1.79, 10.229, 4.036, 2.884, 4.4, 5.0)

    o, g = both(pos, 196.97, ctx, setup=setup)
    o.update()
    g.update()
    assert o.uses_cells()[0]
    no, _ = o.neighbour_list()
    assert no.sum() == 40  # the 20 inside pairs, both ways
    compare_lists(o, g)
    g.destroy()


def test_list_single_atom_and_cluster(ctx):
    from gems_b200 import workloads as W
    for n in (1, 2, 500):
        pos = W.cluster(n, np.random.default_rng(n)) if n > 2 else np.array([[0.0, 0, 0], [2.8, 0, 0]])[:n]
        o, g = both(pos, 196.97, ctx, setup=lambda s: s.set_smatb(*W.SMATB["Au"]))
        o.update()
        g.update()
        compare_lists(o, g)


# ------------------------------------------------------------------ forces
def check_forces(o, g, rms, etol):
    """forces: relative RMS; energies: total per atom and per-atom RMS <= etol,
    largest single-atom deviation <= 5 etol."""
    eo = o.interact()
    eg = g.interact()
    fo, fg = o.force, g.force
    assert relrms(fg, fo) <= rms, relrms(fg, fo)
    d = (g.epot_atoms - o.epot_atoms) * gems.UI_EV
    assert abs(eg - eo) * gems.UI_EV / o.n <= etol, abs(eg - eo) * gems.UI_EV / o.n
    assert np.sqrt(np.mean(d * d)) <= etol, np.sqrt(np.mean(d * d))
    assert np.abs(d).max() <= 5 * etol, np.abs(d).max()


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_smatb_forces_32k(ctx, prec, rms, etol):
    from gems_b200 import workloads as W
    w = W.smatb_bulk()

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        s.set_smatb(*w["smatb"])
    o, g = both(w["pos"], w["mass"], ctx, setup=setup)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_smatb_alloy_cluster(ctx, prec, rms, etol):
    """Two species (Au/Ag cross pair by arithmetic means), free cluster."""
    from gems_b200 import workloads as W
    rng = np.random.default_rng(11)
    pos = W.cluster(800, rng)
    types = (rng.random(800) < 0.4).astype(np.int32)
    mass = np.where(types == 0, W.MASS["Au"], W.MASS["Ag"])
    au, ag = W.SMATB["Au"], W.SMATB["Ag"]
    cross = tuple(0.5 * (a + b) for a, b in zip(au, ag))

    def setup(s):
        s.set_smatb(*au, ti=0, tj=0)
        s.set_smatb(*ag, ti=1, tj=1)
        s.set_smatb(*cross, ti=0, tj=1)
    o, g = both(pos, mass, ctx, types, 2, setup=setup)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_lj_fluid_forces(ctx, prec, rms, etol):
    from gems_b200 import workloads as W
    w = W.lj_fluid()
    rng = np.random.default_rng(3)
    pos = np.mod(w["pos"] + rng.normal(0, 0.05, w["pos"].shape), w["L"][0])

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        e, sg, rc, sh = w["lj"]
        s.set_lj(e, sg, rc, eshift=sh)
        s.set_skin(w["skin"])
    o, g = both(pos, 1.0, ctx, setup=setup)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)


# ------------------------------------------------------------------ half lists
@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_half_list_forces_32k(ctx, prec, rms, etol):
    """A half-list system (Newton on, the serial build's default): its list is
    the reference's half list, entry by entry, and its forces and per-atom
    energies are the full-list oracle's (with the reaction added to j a half
    list gives every atom the same force, density and energy)."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk()

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        s.set_smatb(*w["smatb"])
    o, g = both(w["pos"], w["mass"], ctx, setup=setup)
    g.set_half(True)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)
    oh = O.System(w["pos"], w["mass"])
    setup(oh)
    oh.set_half(True)
    oh.update()
    compare_lists(oh, g)
    g.destroy()


@pytest.mark.parametrize("kind", ["lj", "tersoff", "open_cluster"])
def test_half_list_forces_other_fields(ctx, kind):
    """Half lists under LJ (linked cells), Tersoff (which needs the full set
    of bonds) and an open SMA-TB cluster (O(N^2) lists): FP64 forces against
    the oracle, and the half list against the oracle's."""
    from gems_b200 import workloads as W
    if kind == "lj":
        w = W.lj_fluid()
        rng = np.random.default_rng(3)
        pos, mass = np.mod(w["pos"] + rng.normal(0, 0.05, w["pos"].shape), w["L"][0]), 1.0

        def setup(s):
            s.set_box(w["L"], (True, True, True))
            e, sg, rc, sh = w["lj"]
            s.set_lj(e, sg, rc, eshift=sh)
            s.set_skin(w["skin"])
    elif kind == "tersoff":
        rng = np.random.default_rng(4)
        L = 6 * 5.431
        pos = np.mod(W.diamond(6, 5.431) + rng.normal(0, 0.08, (1728, 3)), L)
        mass = W.MASS["Si"]

        def setup(s):
            s.set_box((L, L, L), (True, True, True))
            s.set_tersoff(W.TERSOFF_SI)
    else:
        pos, mass = W.cluster(300, np.random.default_rng(8)), W.MASS["Au"]

        def setup(s):
            s.set_smatb(*W.SMATB["Au"])
    o, g = both(pos, mass, ctx, setup=setup)
    g.set_half(True)
    check_forces(o, g, RMS_FP64, E_FP64)
    oh = O.System(pos, mass)
    setup(oh)
    oh.set_half(True)
    oh.update()
    compare_lists(oh, g)
    g.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_half_list_md_equals_full_list_md(ctx, prec):
    """The force kernels read the same full list in both list modes, so 200
    Ermak steps of a half-list system equal those of a full-list one, bit for
    bit."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)

    def mk(half):
        g = gems.System(w["pos"], w["mass"], ctx=ctx)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_half(half)
        g.set_precision(prec)
        g.set_ermak(0.002, 1.0, 600.0, seed=3)
        g.interact()
        g.md_steps(200)
        return g
    a, b = mk(False), mk(True)
    np.testing.assert_array_equal(b.pos, a.pos)
    np.testing.assert_array_equal(b.vel, a.vel)
    a.destroy()
    b.destroy()


def _tersoff_crystal(ctx, ncell, sigma, seed):
    """Diamond Si(C) of ncell^3 cells with N(0, sigma) displacements (A)."""
    from gems_b200 import workloads as W
    rng = np.random.default_rng(seed)
    L = ncell * 5.431
    pos = np.mod(W.diamond(ncell, 5.431) + rng.normal(0, sigma, (8 * ncell ** 3, 3)), L)

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
    return both(pos, W.MASS["Si"], ctx, setup=setup)


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_tersoff_forces(ctx, prec, rms, etol):
    """512-atom diamond, displacements of 0.05 A."""
    o, g = _tersoff_crystal(ctx, 4, 0.05, 5)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)
    g.destroy()


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_tersoff_forces_32k(ctx, prec, rms, etol):
    """32768-atom diamond (16^3 cells) with thermal displacements of 0.1 A
    (about the spread of silicon at 1000 K)."""
    o, g = _tersoff_crystal(ctx, 16, 0.1, 6)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)
    g.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_tersoff_forces_reproducible(ctx, prec):
    """The forces are gathered in a fixed order (no atomics): two evaluations
    of the same state, and the same state in a second system, give the same
    bits."""
    _, g = _tersoff_crystal(ctx, 6, 0.1, 8)
    _, h = _tersoff_crystal(ctx, 6, 0.1, 8)
    for s in (g, h):
        s.set_precision(prec)
    g.interact()
    f1, e1 = g.force, g.epot_atoms
    g.set_pos(g.pos)          # dirty: the next call rebuilds and recomputes
    g.interact()
    np.testing.assert_array_equal(g.force, f1)
    np.testing.assert_array_equal(g.epot_atoms, e1)
    h.interact()
    np.testing.assert_array_equal(h.force, f1)
    g.destroy()
    h.destroy()


@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, E_MIXED)])
def test_tersoff_open_clusters(ctx, prec, rms, etol):
    """No box (O(N^2) lists): an isolated atom (no bonds), a dimer (zeta = 0,
    b = chi), a bent trimer, a bond in the cut-off region (R-D < r < R+D) and
    a 40-atom random blob, as one system."""
    from gems_b200 import workloads as W
    rng = np.random.default_rng(9)
    blob = W.diamond(2, 5.431)[:40] + rng.normal(0, 0.08, (40, 3))
    parts = [np.array([[0.0, 0.0, 0.0]]),
             np.array([[0.0, 0.0, 0.0], [2.3, 0.1, 0.0]]),
             np.array([[0.0, 0.0, 0.0], [2.35, 0.0, 0.0], [-0.8, 2.2, 0.1]]),
             np.array([[0.0, 0.0, 0.0], [2.88, 0.05, 0.0], [1.1, 2.1, 0.0]]),
             blob]
    pos = np.concatenate([p + 30.0 * k for k, p in enumerate(parts)])
    o, g = both(pos, W.MASS["Si"], ctx, setup=lambda s: s.set_tersoff(W.TERSOFF_SI))
    g.set_precision(prec)
    check_forces(o, g, rms, etol)
    assert np.all(g.force[0] == 0.0) and g.epot_atoms[0] == 0.0
    g.destroy()


def test_tersoff_batch_equals_alone(ctx):
    """Tersoff crystals of three sizes, 200 NVE steps as one batch equal each
    system's 200 steps alone, bit for bit (mixed precision, 1500 K)."""
    from gems_b200 import workloads as W

    def mk(nc, seed):
        L = nc * 5.431
        pos = W.diamond(nc, 5.431)
        vel = W.maxwell(len(pos), W.MASS["Si"], 1500.0, np.random.default_rng(seed))
        g = gems.System(pos, W.MASS["Si"], ctx=ctx, vel=vel)
        g.set_box((L, L, L), (True, True, True))
        g.set_tersoff(W.TERSOFF_SI)
        g.set_precision(1)
        g.set_vv(0.001)
        g.interact()
        return g
    sizes = (4, 6, 5)
    a = [mk(nc, 60 + k) for k, nc in enumerate(sizes)]
    b = [mk(nc, 60 + k) for k, nc in enumerate(sizes)]
    ctx.batch_md_steps(a, 200)
    for g in b:
        g.md_steps(200)
    for ga, gb in zip(a, b):
        np.testing.assert_array_equal(ga.pos, gb.pos)
        np.testing.assert_array_equal(ga.vel, gb.vel)
        assert ga.nupd == gb.nupd
    for g in a + b:
        g.destroy()


# ------------------------------------------------------------------ golden decks
def gpu_ref_sys(*a, **k):
    """A GPU system with the reference's raw-displacement skin test."""
    g = gems.System(*a, **k)
    g.set_skin_mode(False)
    return g


def test_gpu_xyz_frames(ctx):
    d = decks.xyz_deck()
    g = gpu_ref_sys(d["frames"][0], 12.0, ctx=ctx)
    g.set_box(d["box"], (True, True, True))
    g.set_lj(*d["lj"])
    out = []
    for f in d["frames"]:
        g.set_pos(f)
        out.append(g.interact() * gems.UI_EV)
    assert decks.gems_rule(d["ref"], out) < 1e-6
    np.testing.assert_allclose(out, d["ref"], rtol=2e-7)


@pytest.mark.parametrize("kind", ["lj", "slj"])
def test_gpu_lj_dimer(ctx, kind):
    """lj.gms and slj.gms on the GPU (FP64)."""
    got, ref = decks.lj_dimer_rows(lambda p, m: gpu_ref_sys(p, m, ctx=ctx), gems.UI_EV, kind)
    assert decks.gems_rule(ref[:, 0], got[:, 0]) < 1e-6
    np.testing.assert_allclose(got, ref, atol=2e-7, rtol=1e-6)


@pytest.mark.parametrize("kind", ["wca", "sm1", "feels"])
def test_gpu_lj_family_decks(ctx, kind):
    """wca.gms, sm1.gms and feels.gms on the GPU (FP64) against their golden
    files, and row by row against the oracle."""
    got, ref = decks.lj_family_rows(lambda p, m, t, nt: gpu_ref_sys(p, m, t, nt, ctx=ctx), gems.UI_EV, kind)
    assert got.shape == ref.shape
    assert decks.gems_rule(ref[:, 0], got[:, 0]) < 1e-6
    np.testing.assert_allclose(got, ref, atol=6e-7, rtol=1e-6)
    orc, _ = decks.lj_family_rows(O.System, 1.0 / O.lib().orc_ev_ui(), kind)
    np.testing.assert_allclose(got, orc, atol=1e-12, rtol=1e-9)


# the compressed WCA core puts pair energies of several eV on an atom, of
# which FP32 pair math carries about 6e-8: the mixed energy bound is 4e-6 eV
@pytest.mark.parametrize("prec,rms,etol", [(0, RMS_FP64, E_FP64), (1, RMS_MIXED, 4e-6)])
def test_gpu_wca_feels_fluid(ctx, prec, rms, etol):
    """A dense two-species WCA fluid (2048 atoms, periodic, linked cells)
    where species 1 feels species 0 one-sidedly and an sm1 well binds
    species 1 to itself: forces and per-atom energies against the oracle
    (FP64 and, without sm1, mixed)."""
    rng = np.random.default_rng(21)
    a = 1.6
    k = np.arange(8) * a
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    pos = (np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 1, 3) + base).reshape(-1, 3)
    pos = pos + rng.normal(0.0, 0.05, pos.shape)
    types = np.arange(len(pos)) % 2
    L = 8 * a

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_wca(1.0, 1.0, ti=0, tj=0)
        s.set_wca(0.5, 1.05, ti=1, tj=0)
        s.set_feels(1, 0)
        if prec == 0:
            s.set_sm1(1.0, 1.9, 0.2, ti=1, tj=1)
        else:
            s.set_wca(0.8, 0.95, ti=1, tj=1)
    o, g = both(pos, 39.95, ctx, types, 2, setup=setup)
    g.set_precision(prec)
    check_forces(o, g, rms, etol)
    g.destroy()


def test_gpu_feels_survives_later_pair_setter(ctx):
    """set_feels(1, 0) then set_wca of the same pair again (the reversed
    order): the pair stays one-sided, so the forces equal those of the
    setter-then-feels order, bit for bit."""
    rng = np.random.default_rng(22)
    pos = rng.uniform(0, 9.0, (400, 3))
    pos = pos[np.all(np.linalg.norm(pos[:, None] - pos[None], axis=-1) + 9 * np.eye(400) > 0.9, axis=1)]
    types = (np.arange(len(pos)) % 2).astype(np.int32)

    def mk(again):
        g = gems.System(pos, 39.95, types, 2, ctx=ctx)
        g.set_box((9.0, 9.0, 9.0), (True, True, True))
        g.set_wca(1.0, 1.0, ti=0, tj=0)
        g.set_wca(0.5, 1.05, ti=1, tj=0)
        g.set_feels(1, 0)
        if again:
            g.set_wca(0.5, 1.05, ti=1, tj=0)
        g.set_wca(0.8, 0.95, ti=1, tj=1)
        g.interact()
        return g
    a, b = mk(False), mk(True)
    np.testing.assert_array_equal(b.force, a.force)
    np.testing.assert_array_equal(b.epot_atoms, a.epot_atoms)
    a.destroy()
    b.destroy()


def test_gpu_feels_guards(ctx):
    """One-sided pairs: forces on the feeling type only; no virial, no
    piston; sm1 stays FP64."""
    pos = np.array([[1.0, 1.0, 1.0], [2.0, 1.0, 1.0], [5.0, 5.0, 5.0]])
    g = gpu_ref_sys(pos, 1.008, np.array([0, 1, 1]), 2, ctx=ctx)
    g.set_box((10.0, 10.0, 10.0), (True, True, True))
    g.set_wca(1.0, 0.95, ti=1, tj=0)
    g.set_feels(1, 0)
    g.interact()
    f = g.force
    assert np.all(f[0] == 0.0) and f[1, 0] > 0.0 and np.all(f[2] == 0.0)
    with pytest.raises(gems.GemsGpuError):
        g.set_virial(True)
    with pytest.raises(gems.GemsGpuError):
        g.set_lgf(0.002, 300.0, 1.0, 1.0, 1.0, 10.0)
    h = gpu_ref_sys(pos, 1.008, ctx=ctx)
    h.set_sm1(1.0, 2.0, 0.01)
    with pytest.raises(gems.GemsGpuError):
        h.set_precision(gems.PREC_MIXED)
    g.destroy()
    h.destroy()


def test_gpu_smatb_bulk_ermak_parity_stream(ctx):
    d = decks.bulk_deck()
    g = gpu_ref_sys(d["pos"], d["mass"], ctx=ctx)
    smatb_bulk_setup(g)
    g.set_ermak(d["dt"], d["gamma"], d["temp"])
    rows = decks.ermak_parity_run(g, O.Rng(d["seed"]), d["nsteps"], d["each"])
    ref = d["ref"]
    assert decks.gems_rule(ref[:, 0], rows[:, 0] * gems.UI_EV) < 1e-6
    np.testing.assert_allclose(rows[:, :3] * gems.UI_EV, ref, rtol=2e-6)


def test_gpu_nve_plj(ctx):
    pos, vel, types, mass, box, _ = decks.he_ne_setup(O)
    g = gpu_ref_sys(pos, mass, types, 2, ctx=ctx, vel=vel)
    g.set_box(box, (True, True, True))
    decks.apply_plj(g)
    g.set_vv(0.002)
    r = g.dinamica(5000, 100)
    ref = np.array(decks.golden()["nve_energy"])
    assert decks.gems_rule(ref[:, 0], r[:, 0]) < 1e-6
    np.testing.assert_allclose(r[:, 1:3], ref[:, 1:3], rtol=1e-5)


def _he_ne_gpu(ctx):
    pos, vel, types, mass, box, _ = decks.he_ne_setup(O)
    g = gpu_ref_sys(pos, mass, types, 2, ctx=ctx, vel=vel)
    g.set_box(box, (True, True, True))
    decks.apply_plj(g)
    return g


def test_gpu_nve_pred_corr(ctx):
    """pred_corr_5.gms on the GPU: the same gas under the fifth-order
    Nordsieck predictor-corrector, against its golden file."""
    g = _he_ne_gpu(ctx)
    g.set_pred_corr(0.002)
    r = g.dinamica(5000, 100)
    ref = np.array(decks.golden()["nve_pc5_energy"])
    assert decks.gems_rule(ref[:, 0], r[:, 0]) < 1e-6
    np.testing.assert_allclose(r[:, 1:3], ref[:, 1:3], rtol=1e-5)
    g.destroy()


def test_gpu_pred_corr_derivatives_and_resume(ctx):
    """The predictor-corrector's derivatives acel..acel4 after 200 steps
    match the oracle's, read from GEMS's .chp file; a system resumed from
    the file written at step 100 continues the unbroken trajectory."""
    pos, vel, types, mass, box, _ = decks.he_ne_setup(O)
    n = len(pos)
    s = O.System(pos, mass, types, 2)
    s.set_box(box, (True, True, True))
    s.set_vel(vel)
    decks.apply_plj(s)
    s.set_pred_corr(0.002)
    s.dinamica(200, 100)
    want = s.derivs()
    g = _he_ne_gpu(ctx)
    g.set_pred_corr(0.002)
    g.dinamica(100, 100)
    chp = g.write_gems_chp(step=100, nsteps=100)
    ck = g.checkpoint()
    g.dinamica(100, 100)
    got = decks.chp_atoms(g.write_gems_chp(step=200, nsteps=200), n)
    np.testing.assert_allclose(got[0], s.pos, rtol=0, atol=1e-9)
    for k in range(4):
        scale = np.abs(want[k]).max()
        assert scale > 0.0
        np.testing.assert_allclose(got[2 + k], want[k], rtol=1e-6, atol=1e-8 * scale)
    h = gpu_ref_sys(np.zeros_like(pos), mass, types, 2, ctx=ctx)
    h.set_box(box, (True, True, True))
    decks.apply_plj(h)
    h.set_pred_corr(0.002)
    assert h.read_gems_chp(chp)["step"] == 100
    h.dinamica(100, 100)
    np.testing.assert_allclose(h.pos, g.pos, rtol=0, atol=1e-9)
    np.testing.assert_allclose(h.vel, g.vel, rtol=1e-9, atol=1e-12)
    # the library's own checkpoint carries the derivatives too
    k = gpu_ref_sys(np.zeros_like(pos), mass, types, 2, ctx=ctx)
    k.set_box(box, (True, True, True))
    decks.apply_plj(k)
    k.set_pred_corr(0.002)
    k.restore(ck)
    k.dinamica(100, 100)
    np.testing.assert_allclose(k.pos, g.pos, rtol=0, atol=1e-9)
    g.destroy()
    h.destroy()
    k.destroy()


def test_gpu_brownian_parity_stream(ctx):
    """examples/NVT/brownian.gms (the gas, tempgdist 300, `evolve brownian
    300 10`) on the oracle's LCG stream: 500 steps on the device against
    the oracle's own run, row by row."""
    pos, vel, types, mass, box, rng_g = decks.he_ne_setup(O)
    g = _he_ne_gpu(ctx)
    g.set_brownian(0.002, 300.0, 10.0)
    rows = decks.ermak_parity_run(g, rng_g, 500, 100)
    _, _, _, _, _, rng_o = decks.he_ne_setup(O)
    s = O.System(pos, mass, types, 2)
    s.set_box(box, (True, True, True))
    s.set_vel(vel)
    decks.apply_plj(s)
    s.set_brownian(0.002, 300.0, 10.0, rng_o)
    want = s.dinamica(500, 100)
    np.testing.assert_allclose(rows[:, :3] * gems.UI_EV, want[:, :3], rtol=1e-9)
    np.testing.assert_allclose(rows[:, 3], want[:, 3], rtol=1e-9)
    np.testing.assert_allclose(g.pos, s.pos, rtol=0, atol=1e-9)
    g.destroy()


def test_gpu_brownian_philox(ctx):
    """Brownian dynamics on the device stream: the displacement noise of a
    step has variance 2 kB T dt / (gamma m) per coordinate (force-free
    atoms: a dilute gas far beyond the cut-off)."""
    k = np.arange(16) * 25.0 + 5.0
    pos = np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3)
    g = gpu_ref_sys(pos, 4.0032, ctx=ctx)
    g.set_box((400.0, 400.0, 400.0), (True, True, True))
    g.set_lj(1e-6, 1.0, 1.5)
    dt, temp, gama = 0.002, 300.0, 10.0
    g.set_brownian(dt, temp, gama, seed=77)
    g.dinamica(1, 1)
    v = g.vel
    d = v * dt
    kB_ui = O.lib().orc_kB_ui()
    var = 2.0 * kB_ui * temp * dt / gama / 4.0032
    assert abs(d.var() / var - 1.0) < 0.05
    assert abs(d.mean()) < 4.0 * np.sqrt(var / d.size)
    g.destroy()


@pytest.mark.parametrize("upto", [None, 0.02])
@pytest.mark.parametrize("drift", [0.0, 500.0])
def test_gpu_scalvel_matches_oracle(ctx, upto, drift):
    """scalvel (and scalvel_after with a narrow band) after velocity Verlet
    on the gas of v_verlet.gms, toward 250 K: the device's md_steps rows
    against the oracle's.  drift (A/ps, about 70 thermal speeds) is added to
    every velocity: the temperature is the kinetic energy about the centre of
    mass, which must not lose digits to the drift."""
    pos, vel, types, mass, box, _ = decks.he_ne_setup(O)
    vel = vel + drift * np.array([0.6, -0.48, 0.64])
    g = _he_ne_gpu(ctx)
    g.set_vel(vel)
    g.set_vv(0.002)
    g.set_scalvel(250.0, 10, upto)
    rows = g.dinamica(400, 50)
    s = O.System(pos, mass, types, 2)
    s.set_box(box, (True, True, True))
    s.set_vel(vel)
    decks.apply_plj(s)
    s.set_vv(0.002)
    s.set_scalvel(250.0, 10, upto)
    want = s.dinamica(400, 50)
    np.testing.assert_allclose(rows[:, :4], want[:, :4], rtol=1e-8)
    assert abs(rows[-1, 3] - 250.0) < 0.1 * 250.0
    g.destroy()


def test_gpu_andersen_statistics(ctx):
    """andersen after velocity Verlet, force-free atoms: with nu dt = 1/4 a
    quarter of the atoms collide per step; with nu dt = 1 every atom does
    and m v^2 averages the reference's kB T / (3N)^2 per coordinate."""
    k = np.arange(16) * 25.0 + 5.0
    pos = np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3)
    n = len(pos)
    vel = np.tile([1e-3, 2e-3, 3e-3], (n, 1))
    g = gpu_ref_sys(pos, 4.0032, ctx=ctx, vel=vel)
    g.set_box((400.0, 400.0, 400.0), (True, True, True))
    g.set_lj(1e-6, 1.0, 1.5)
    g.set_vv(0.002)
    g.set_andersen(300.0, 0.25 / 0.002, seed=5)
    g.dinamica(1, 1)
    hit = np.any(g.vel != vel, axis=1)
    assert abs(hit.mean() - 0.25) < 0.03
    g.set_andersen(300.0, 1.0 / 0.002, seed=6)
    kB_ui = O.lib().orc_kB_ui()
    want = kB_ui * 300.0 / (3.0 * n) ** 2
    m2 = []
    for _ in range(3):
        g.dinamica(1, 1)
        m2.append((g.vel ** 2 * 4.0032).ravel())
    assert abs(np.concatenate(m2).mean() / want - 1.0) < 0.05
    g.clear_thermostat()
    g.destroy()


def test_gpu_nvt_plj_parity_stream(ctx):
    pos, vel, types, mass, box, rng = decks.he_ne_setup(O)
    g = gpu_ref_sys(pos, mass, types, 2, ctx=ctx, vel=vel)
    g.set_box(box, (True, True, True))
    decks.apply_plj(g)
    g.set_ermak(0.002, 10.0, 300.0)
    rows = decks.ermak_parity_run(g, rng, 10000, 100)
    ref = np.array(decks.golden()["nvt_energy"])
    assert decks.gems_rule(ref[:, 0], rows[:, 0] * gems.UI_EV) < 1e-6
    np.testing.assert_allclose(rows[:, 3], ref[:, 3], rtol=1e-5)


# ------------------------------------------------------------------ engine invariants
@pytest.mark.parametrize("integ", ["ermak", "vv"])
@pytest.mark.parametrize("prec", [0, 1])
def test_md_steps_equals_stepwise(ctx, integ, prec):
    """The captured md_steps loop (step_b and the next step_a fused into one
    kernel) gives the trajectory of separate step_a / interact / step_b calls
    bit for bit."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=8)
    vel = W.maxwell(len(w["pos"]), w["mass"], 600.0, np.random.default_rng(3))
    sys = []
    for _ in range(2):
        g = gems.System(w["pos"], w["mass"], ctx=ctx, vel=vel)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_precision(prec)
        if integ == "ermak":
            g.set_ermak(w["dt"], w["gamma"], w["temp"], seed=99)
        else:
            g.set_vv(w["dt"])
        g.interact()
        sys.append(g)
    sys[0].md_steps(120)
    for _ in range(120):
        sys[1].stepa()
        sys[1].interact()
        sys[1].stepb()
    np.testing.assert_array_equal(sys[0].pos, sys[1].pos)
    np.testing.assert_array_equal(sys[0].vel, sys[1].vel)
    assert sys[0].nupd == sys[1].nupd
    for g in sys:
        g.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_md_steps_equals_stepwise_large_tersoff(ctx, prec):
    """A 636,056-atom Tersoff Si crystal (43^3 diamond cells, 1000 K): on a
    system this large the captured loop's integrator kernel takes two atoms
    per thread and merges the skin test over half as many blocks; the
    trajectory equals that of separate step_a / interact / step_b calls bit
    for bit over 60 velocity-Verlet steps, list rebuilds included."""
    from gems_b200 import workloads as W
    pos = W.diamond(43, 5.431)
    L = 43 * 5.431
    vel = W.maxwell(len(pos), W.MASS["Si"], 1000.0, np.random.default_rng(4))
    sys = []
    for _ in range(2):
        g = gems.System(pos, W.MASS["Si"], ctx=ctx, vel=vel)
        g.set_box((L, L, L), (True, True, True))
        g.set_tersoff(W.TERSOFF_SI)
        g.set_skin(1.0)
        g.set_precision(prec)
        g.set_vv(0.001)
        g.interact()
        sys.append(g)
    sys[0].md_steps(60)
    for _ in range(60):
        sys[1].stepa()
        sys[1].interact()
        sys[1].stepb()
    np.testing.assert_array_equal(sys[0].pos, sys[1].pos)
    np.testing.assert_array_equal(sys[0].vel, sys[1].vel)
    assert sys[0].nupd == sys[1].nupd >= 2
    for g in sys:
        g.destroy()


def test_batch_state_transfer_equals_per_system_calls(ctx):
    """gemsgpu_batch_set_state / _get_state move the same bytes as the
    per-system calls, and a run after a batched upload equals one after
    per-system uploads."""
    from gems_b200 import workloads as W
    sm, m = W.SMATB["Au"], W.MASS["Au"]
    cl = [W.cluster(n, np.random.default_rng(n)) for n in (40, 200, 90)]
    rng = np.random.default_rng(1)
    runs = []
    for batched in (False, True):
        ss = []
        for p in cl:
            g = gems.System(np.zeros_like(p), m, ctx=ctx)
            g.set_smatb(*sm)
            g.set_ermak(0.002, 1.0, 400.0, seed=3)
            ss.append(g)
        vel = [W.maxwell(len(p), m, 400.0, np.random.default_rng(len(p))) for p in cl]
        if batched:
            ctx.batch_set_state(ss, [np.ascontiguousarray(p) for p in cl], [np.ascontiguousarray(v) for v in vel])
        else:
            for g, p, v in zip(ss, cl, vel):
                g.set_pos(p)
                g.set_vel(v)
        for g, p, v in zip(ss, cl, vel):
            np.testing.assert_array_equal(g.pos, p)
            np.testing.assert_array_equal(g.vel, v)
        ctx.batch_md_steps(ss, 60)
        pos_out = [np.empty(3 * g.n) for g in ss]
        vel_out = [np.empty(3 * g.n) for g in ss]
        ep, ek, t = ctx.batch_get_state(ss, pos_out, vel_out)
        e_ref = ctx.batch_energy(ss)
        for g, po, vo in zip(ss, pos_out, vel_out):
            np.testing.assert_array_equal(po.reshape(-1, 3), g.pos)
            np.testing.assert_array_equal(vo.reshape(-1, 3), g.vel)
        np.testing.assert_array_equal(ep, e_ref[0])
        runs.append(pos_out)
        for g in ss:
            g.destroy()
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)


def test_skin_modes_same_trajectory(ctx):
    """The minimum-image skin test skips the rebuilds that wrapped atoms
    trigger in the reference's test, without changing the dynamics."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=8)
    runs = []
    for mic in (False, True):
        g = gems.System(w["pos"], w["mass"], ctx=ctx)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_skin_mode(mic)
        g.set_vv(0.002)
        g.interact()
        g.md_steps(200)
        runs.append((g.nupd, g.pos, g.energy()))
    (n_ref, p_ref, e_ref), (n_mic, p_mic, e_mic) = runs
    assert n_mic < n_ref
    d = p_mic - p_ref
    d -= w["L"][0] * np.round(d / w["L"][0])
    assert np.abs(d).max() < 1e-9
    assert abs(e_mic[0] - e_ref[0]) / len(p_ref) < 1e-10


@pytest.mark.parametrize("prec", [0, 1])
def test_launch_shapes_agree(ctx, prec):
    """Every lanes-per-atom / constant-placement shape the autotuner may pick
    gives the same forces within the precision's tolerance."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        s.set_smatb(*w["smatb"])
    o, g = both(w["pos"], w["mass"], ctx, setup=setup)
    g.set_precision(prec)
    o.interact()
    fo = o.force
    for lanes in (1, 2, 4, 8, 16, 32):
        for variant in (0, 1, 2, 3, 6, 7):
            g.set_lanes(lanes, variant)
            g.interact()
            assert relrms(g.force, fo) <= (RMS_FP64 if prec == 0 else RMS_MIXED)
    k, v, ms = g.autotune(3)
    assert k in (1, 2, 4, 8, 16, 32) and v in (0, 1, 2, 3, 6, 7) and ms > 0


def _cluster_replicas(ctx, nrep, temps, seed0=7):
    from gems_b200 import workloads as W
    pos = W.cluster(147, np.random.default_rng(3))
    reps = []
    for k in range(nrep):
        g = gems.System(pos + np.random.default_rng(seed0 + k).normal(0, 0.05, pos.shape), W.MASS["Au"],
                        ctx=ctx)
        g.set_smatb(*W.SMATB["Au"])
        g.set_ermak(0.002, 1.0, temps[k], seed=seed0 + k)
        reps.append(g)
    return reps


def test_replica_exchange_rule(ctx):
    """The GPU exchange follows parallel_tempering2's pairing and Metropolis
    rule (restated here from the replicas' energies and the same uniforms)
    and swaps temperature labels with a velocity rescale."""
    nrep = 8
    temps = 200.0 * (900.0 / 200.0) ** (np.arange(nrep) / (nrep - 1))
    reps = _cluster_replicas(ctx, nrep, temps)
    ctx.batch_md_steps(reps, 200)
    order = list(reps)
    rng = np.random.default_rng(0)
    kB = 8.617385e-05
    for rnd in range(1, 7):
        ep, _, _ = ctx.batch_energy(order)
        vel_before = {s.sid: s.vel for s in order}
        u = rng.random(nrep)
        expect = list(order)
        par = 1 if rnd % 2 == 0 else -1
        for k in range(nrep):
            p = k + par if k % 2 == 0 else k - par
            if p < 0 or p >= nrep or p < k:
                continue
            du = (ep[p] - ep[k]) * (1.0 / (kB * temps[k]) - 1.0 / (kB * temps[p]))
            if du <= 0 or u[k] < np.exp(-du):
                expect[k], expect[p] = expect[p], expect[k]
        prev = [s.sid for s in order]
        order, acc = ctx.replica_exchange(order, temps, rnd, uniforms=u)
        assert [s.sid for s in order] == [s.sid for s in expect]
        for k, s in enumerate(order):
            k_old = prev.index(s.sid)
            np.testing.assert_allclose(s.vel, vel_before[s.sid] * np.sqrt(temps[k] / temps[k_old]), rtol=1e-13)
        ctx.batch_md_steps(order, 50)
    assert sorted(s.sid for s in order) == sorted(s.sid for s in reps)


def test_replica_exchange_identical_replicas_always_swap(ctx):
    temps = [300.0, 400.0, 500.0, 600.0]
    reps = _cluster_replicas(ctx, 4, temps, seed0=50)
    from gems_b200 import workloads as W
    pos = W.cluster(147, np.random.default_rng(3))
    for g in reps:
        g.set_pos(pos)
    for g in reps:
        g.interact()
    v0 = {g.sid: g.vel for g in reps}
    order, acc = ctx.replica_exchange(reps, temps, 2, seed=3)
    assert acc == 2  # pairs (0,1) and (2,3): equal energies, always accepted
    assert [s.sid for s in order] == [reps[1].sid, reps[0].sid, reps[3].sid, reps[2].sid]
    # velocities rescaled by sqrt(T_new / T_old)
    np.testing.assert_allclose(order[0].vel, v0[reps[1].sid] * np.sqrt(300.0 / 400.0), rtol=1e-14)
    np.testing.assert_allclose(order[3].vel, v0[reps[2].sid] * np.sqrt(600.0 / 500.0), rtol=1e-14)


def test_replica_exchange_driver_equals_context_call(ctx):
    """The multi-rank driver (here one rank) takes the same decisions as
    gemsgpu_replica_exchange and leaves the same temperatures and velocities."""
    from gems_b200.remd import ReplicaExchange
    nrep = 6
    temps = 250.0 * (800.0 / 250.0) ** (np.arange(nrep) / (nrep - 1))
    a = _cluster_replicas(ctx, nrep, temps, seed0=21)
    b = _cluster_replicas(ctx, nrep, temps, seed0=21)
    rex = ReplicaExchange(ctx, b, temps, seed=13)
    order = list(a)
    acc_a = acc_b = 0
    for rnd in range(1, 9):
        ctx.batch_md_steps(a, 40)
        ctx.batch_md_steps(b, 40)
        order, acc = ctx.replica_exchange(order, temps, rnd, seed=13)
        acc_a += acc
        acc_b += rex.exchange(rnd)
    assert acc_a == acc_b and acc_a > 0
    t_a = {s.sid: temps[k] for k, s in enumerate(order)}
    np.testing.assert_array_equal(rex.local_temperatures(), [t_a[s.sid] for s in a])
    for sa, sb in zip(a, b):
        np.testing.assert_array_equal(sa.vel, sb.vel)
        np.testing.assert_array_equal(sa.pos, sb.pos)
    for g in a + b:
        g.destroy()


def test_fire_single_cluster_vs_oracle(ctx):
    """FIRE (the intent of src/FIRE.f90 with its defects fixed) relaxes a
    perturbed 55-atom Au cluster to the oracle's minimum."""
    from gems_b200 import workloads as W
    pos = W.cluster(55, np.random.default_rng(21), jitter=0.12)
    o = O.System(pos, W.MASS["Au"])
    o.set_smatb(*W.SMATB["Au"])
    o.set_fire(0.002, 0.02)
    it_o, fm_o = o.fire_relax(1e-3, 5000)
    g = gems.System(pos, W.MASS["Au"], ctx=ctx)
    g.set_smatb(*W.SMATB["Au"])
    g.set_fire(0.002, 0.02)
    it_g = ctx.batch_fire([g], 1e-3, 5000)[0]
    assert fm_o < 1e-3 and g.fmax() < 1e-3
    eo = o.epot_sum() * gems.UI_EV / 55
    eg = g.energy()[0] / 55
    assert abs(eo - eg) < 1e-6, (eo, eg)
    assert abs(it_g - it_o) <= max(50, 0.2 * it_o)


def test_fire_batch_equals_alone(ctx):
    """Uneven clusters relaxed in one batch give bit-identical results to the
    same clusters relaxed one at a time."""
    from gems_b200 import workloads as W
    sizes = [13, 80, 300, 38]
    cl = [W.cluster(n, np.random.default_rng(100 + n), jitter=0.1) for n in sizes]

    def mk(p):
        g = gems.System(p, W.MASS["Au"], ctx=ctx)
        g.set_smatb(*W.SMATB["Au"])
        g.set_precision(gems.PREC_MIXED)
        g.set_lanes(4, 1)
        g.set_fire(0.002, 0.02)
        return g

    batch = [mk(p) for p in cl]
    it_b = ctx.batch_fire(batch, 1e-3, 3000)
    for p, gb, itb in zip(cl, batch, it_b):
        ga = mk(p)
        it_a = ctx.batch_fire([ga], 1e-3, 3000)[0]
        assert it_a == itb
        np.testing.assert_array_equal(ga.pos, gb.pos)
        assert ga.energy()[0] == gb.energy()[0]
        ga.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_stale_list_pairs_entering_the_cutoff(ctx, prec):
    """Between list builds the force kernels visit only the band-ordered
    entries that can have come within the cut-off (the skin test's bound on
    how far pairs moved).  A periodic Au crystal is displaced by up to 0.24 A
    per atom without a rebuild, so pairs built outside rce move inside it;
    the forces still match the oracle's full-list sums."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)
    L = np.array(w["L"])

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        s.set_smatb(*w["smatb"])
    o, g = both(w["pos"], w["mass"], ctx, setup=setup)
    g.set_precision(prec)
    o.interact()
    g.interact()
    n0 = g.nupd
    rng = np.random.default_rng(11)
    step = rng.normal(size=w["pos"].shape)
    step *= (0.24 * rng.random(len(step)) / np.linalg.norm(step, axis=1))[:, None]
    moved = np.mod(w["pos"] + step, L)
    rce = w["smatb"][6]
    d0 = w["pos"][None, :, :] - w["pos"][:, None, :]
    d1 = moved[None, :, :] - moved[:, None, :]
    d0 -= L * np.round(d0 / L)
    d1 -= L * np.round(d1 / L)
    r0, r1 = np.linalg.norm(d0, axis=2), np.linalg.norm(d1, axis=2)
    assert np.sum((r0 > rce) & (r1 < rce)) > 0  # pairs that entered the cut-off
    o.set_pos(moved)
    g.set_pos(moved)
    o.interact()
    g.interact()
    assert g.nupd == n0  # no rebuild: the stale list was used
    assert relrms(g.force, o.force) <= (RMS_FP64 if prec == 0 else RMS_MIXED)
    g.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_tersoff_stale_list_bonds_entering_the_cutoff(ctx, prec):
    """The Tersoff bond scan stops at the entries that can have come within
    R+D (the skin test's bound on how far pairs moved).  A diamond with its
    second shell squeezed to just beyond R+D is displaced
    without a rebuild (a few atoms by 0.45 A, the rest by up to 0.12 A) so
    that second-shell pairs become bonds; the forces still match the oracle's
    fresh full-list sums."""
    from gems_b200 import workloads as W
    a = 4.45          # second shell at a/sqrt(2) = 3.15 A, first at 1.93 A
    L = 6 * a
    rng = np.random.default_rng(12)
    pos0 = np.mod(W.diamond(6, a) + rng.normal(0, 0.01, (1728, 3)), L)

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
        s.set_skin(1.0)
    o, g = both(pos0, W.MASS["Si"], ctx, setup=setup)
    g.set_precision(prec)
    o.interact()
    g.interact()
    n0 = g.nupd
    step = rng.normal(size=pos0.shape)
    mag = 0.12 * rng.random(len(step))
    mag[rng.choice(len(step), 8, replace=False)] = 0.45
    step *= (mag / np.linalg.norm(step, axis=1))[:, None]
    moved = np.mod(pos0 + step, L)
    d0 = pos0[None, :, :] - pos0[:, None, :]
    d1 = moved[None, :, :] - moved[:, None, :]
    d0 -= L * np.round(d0 / L)
    d1 -= L * np.round(d1 / L)
    r0, r1 = np.linalg.norm(d0, axis=2), np.linalg.norm(d1, axis=2)
    assert np.sum((r0 > 3.0) & (r1 <= 3.0)) > 0   # pairs that became bonds
    o.set_pos(moved)
    g.set_pos(moved)
    o.interact()
    g.interact()
    assert g.nupd == n0  # no rebuild: the stale list was used
    check_forces(o, g, RMS_FP64 if prec == 0 else RMS_MIXED, E_FP64 if prec == 0 else E_MIXED)
    g.destroy()


def test_batched_graph_branches_equal_alone(ctx):
    """A batch runs as one graph branch per system (its own steps,
    conditional rebuilds and force passes), so systems overlap on the GPU.
    Three periodic crystals of different sizes, hot enough to rebuild at
    different steps: 300 batched Ermak steps equal each system's 300 steps
    run alone, bit for bit, rebuild counts included."""
    from gems_b200 import workloads as W

    def mk(nc, seed):
        w = W.smatb_bulk(ncell=nc)
        vel = W.maxwell(len(w["pos"]), w["mass"], 900.0, np.random.default_rng(seed))
        g = gems.System(w["pos"], w["mass"], ctx=ctx, vel=vel)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_precision(1)
        g.set_lanes(2, 1)
        g.set_ermak(w["dt"], w["gamma"], 900.0, seed=seed)
        g.interact()
        return g
    sizes = (5, 7, 6)
    a = [mk(nc, 20 + k) for k, nc in enumerate(sizes)]
    b = [mk(nc, 20 + k) for k, nc in enumerate(sizes)]
    ctx.batch_md_steps(a, 300)
    for g in b:
        g.md_steps(300)
    for ga, gb in zip(a, b):
        np.testing.assert_array_equal(ga.pos, gb.pos)
        np.testing.assert_array_equal(ga.vel, gb.vel)
        assert ga.nupd == gb.nupd
    assert len({g.nupd for g in a}) > 1 or all(g.nupd > 1 for g in a)
    for g in a + b:
        g.destroy()


def test_large_batch_grouped_branches_equal_alone(ctx):
    """Batches of more than 16 systems run as 16 branches of consecutive
    systems; 18 uneven crystals, 100 batched Ermak steps, equal to each
    system alone, bit for bit."""
    from gems_b200 import workloads as W

    def mk(nc, seed):
        w = W.smatb_bulk(ncell=nc)
        vel = W.maxwell(len(w["pos"]), w["mass"], 900.0, np.random.default_rng(seed))
        g = gems.System(w["pos"], w["mass"], ctx=ctx, vel=vel)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_precision(1)
        g.set_lanes(4, 1)
        g.set_ermak(w["dt"], w["gamma"], 900.0, seed=seed)
        g.interact()
        return g
    sizes = [4, 5, 6] * 6
    a = [mk(nc, 40 + k) for k, nc in enumerate(sizes)]
    b = [mk(nc, 40 + k) for k, nc in enumerate(sizes)]
    ctx.batch_md_steps(a, 100)
    for g in b:
        g.md_steps(100)
    for ga, gb in zip(a, b):
        np.testing.assert_array_equal(ga.pos, gb.pos)
        np.testing.assert_array_equal(ga.vel, gb.vel)
        assert ga.nupd == gb.nupd
    for g in a + b:
        g.destroy()
