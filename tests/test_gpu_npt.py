"""Constant pressure on the GPU: slj forces with the pair virial, and the
G-JF piston (set_lgf / lgf_stepa / lgf_stepb, src/Integration.F90:486-650)
against the oracle and the examples/NPT/lgf.gms golden files."""
import numpy as np
import pytest

import decks
from oracle import oracle as O

gems = pytest.importorskip("gems_b200")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gems.Context()
    yield c
    c.close()


def _gpu(ctx, d, pos=None, seed=12345, skin=None):
    g = gems.System(d["pos"] if pos is None else pos, d["mass"], ctx=ctx)
    g.set_skin_mode(False)  # the reference's raw-displacement skin test
    if skin is not None:
        g.set_skin(skin)
    g.set_box(d["box"], (True, True, True))
    g.set_slj(*d["slj"])
    g.set_lgf(d["dt"], d["temp"], d["press_atm"], d["pgama0"], d["pgamav"], d["pmass"], seed=seed)
    return g


def _oracle(d, pos=None, skin=None):
    s = O.System(d["pos"] if pos is None else pos, d["mass"])
    if skin is not None:
        s.set_skin(skin)
    rng = O.Rng(d["seed"])
    decks.npt_setup(s, d, rng)
    return s, rng


def _feed(g, nrm):
    g.set_lgf_normals(nrm)


def test_slj_forces_and_virial_equal_oracle(ctx):
    """One interact of the lgf.gms crystal, displaced: forces, energy and
    virial."""
    d = decks.npt_lgf_deck()
    rng = np.random.default_rng(5)
    pos = d["pos"] + rng.normal(0.0, 0.05, d["pos"].shape)
    s, _ = _oracle(d, pos)
    s.interact()
    g = _gpu(ctx, d, pos)
    g.interact()
    f_ref = s.force
    np.testing.assert_allclose(g.force, f_ref, rtol=0, atol=1e-10 * np.abs(f_ref).max())
    assert abs(g.epot_sum() - s.epot_sum()) < 1e-10 * abs(s.epot_sum())
    np.testing.assert_allclose(g.virial_ev(), s.virial_ev(), rtol=1e-10, atol=1e-8)
    g.destroy()


def test_slj_mixed_forces_and_virial(ctx):
    """slj in mixed precision (FP32 pair math with the quartic-octic tail,
    FP64 accumulation): forces to 1e-5 relative RMS, energy to 1e-6 eV per
    atom and the virial to 1e-5 of its largest component against the oracle."""
    d = decks.npt_lgf_deck()
    rng = np.random.default_rng(6)
    pos = d["pos"] + rng.normal(0.0, 0.05, d["pos"].shape)
    s, _ = _oracle(d, pos)
    s.interact()
    g = _gpu(ctx, d, pos)
    g.set_precision(1)
    g.interact()
    f_ref = s.force
    assert np.linalg.norm(g.force - f_ref) / np.linalg.norm(f_ref) <= 1e-5
    assert abs(g.epot_sum() - s.epot_sum()) * O.UI_EV / len(pos) <= 1e-6
    ref = s.virial_ev()
    np.testing.assert_allclose(g.virial_ev(), ref, rtol=0, atol=1e-5 * np.abs(ref).max())
    g.destroy()


def test_lgf_trajectory_equals_oracle(ctx):
    """100 piston steps with the oracle's normals fed to the device: energy,
    pressure, virial and box at every 10th step."""
    d = decks.npt_lgf_deck()
    s, rng_o = _oracle(d)
    E0, P0, V0 = decks.npt_run(s, d, rng_o)
    g = _gpu(ctx, d)
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(d["seed"]), feed=_feed)
    np.testing.assert_allclose(E1, E0, rtol=1e-9)
    np.testing.assert_allclose(P1, P0, rtol=1e-8, atol=1e-3)
    np.testing.assert_allclose(V1, V0, rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(g.box_now(), s.box_now(), rtol=1e-12)
    g.destroy()


def test_lgf_deck_golden(ctx):
    """lgf.gms on the GPU against Energy.lgf.dat, Press.lgf.dat and
    Viri.lgf.dat (7 significant digits)."""
    d = decks.npt_lgf_deck()
    g = _gpu(ctx, d)
    E, P, V = decks.npt_run(g, d, O.Rng(d["seed"]), feed=_feed)
    E[:, :3] *= O.UI_EV
    assert decks.gems_rule(d["ref_energy"][:, 0], E[:, 0]) < 1e-6
    np.testing.assert_allclose(E, d["ref_energy"], rtol=2e-6)
    np.testing.assert_allclose(P, d["ref_press"], rtol=2e-6, atol=1e-2)
    np.testing.assert_allclose(V, d["ref_virial"], rtol=2e-6, atol=1e-6)
    g.destroy()


@pytest.mark.parametrize("prec", [0, 1])
def test_lgf_md_steps_equals_stepwise(ctx, prec):
    """The captured md_steps loop (piston kernel, half steps, conditional
    rebuilds) gives the trajectory of separate step calls bit for bit, with
    the device's own noise, in FP64 and in mixed precision (where the
    fixed-point frame follows the moving box)."""
    d = decks.npt_lgf_deck()
    a = _gpu(ctx, d, seed=7)
    b = _gpu(ctx, d, seed=7)
    a.set_precision(prec)
    b.set_precision(prec)
    a.interact()
    b.interact()
    a.md_steps(120)
    for _ in range(120):
        b.stepa()
        b.interact()
        b.stepb()
    np.testing.assert_array_equal(a.pos, b.pos)
    np.testing.assert_array_equal(a.vel, b.vel)
    np.testing.assert_array_equal(a.box_now(), b.box_now())
    assert a.nupd == b.nupd
    assert abs(a.box_now()[0] - d["box"][0]) > 1e-3
    a.destroy()
    b.destroy()


def test_lgf_checkpoint_resume(ctx):
    """lgf_flex_a/b style: 60 steps, checkpoint, a fresh system restored from
    it runs 60 more; the straight 120-step run ends at the same state (the
    resumed interact rebuilds the list, so the pair sums may round in
    another order)."""
    d = decks.npt_lgf_deck()
    a = _gpu(ctx, d, seed=11)
    a.md_steps(120)
    b = _gpu(ctx, d, seed=11)
    b.md_steps(60)
    chp = b.checkpoint()
    b.destroy()
    c = _gpu(ctx, d, pos=np.zeros_like(d["pos"]), seed=11)
    c.restore(chp)
    c.md_steps(60)
    np.testing.assert_allclose(c.box_now(), a.box_now(), rtol=1e-10)
    np.testing.assert_allclose(c.pos, a.pos, rtol=0, atol=1e-8)
    np.testing.assert_allclose(c.vel, a.vel, rtol=0, atol=1e-8 * np.abs(a.vel).max())
    a.destroy()
    c.destroy()


def test_lgf_cell_grid_follows_the_box(ctx):
    """A crystal of 12^3 fcc cells (6912 atoms) whose box is 5.01 list
    cut-offs long, compressed at 1 e0/r0^3: between list builds the box
    shrinks below five cut-offs, so the linked-cell grid must drop from 5^3
    to 4^3 cells (the device re-plans it within the cells allocated, the
    oracle recomputes it at each list update), and the trajectory stays the
    oracle's."""
    d = decks.npt_lgf_deck()
    f = np.sqrt(2.0)
    L0 = 12.0 * f
    rc = 1.959794718597571  # slj cut-off of (1, 2^(-1/6), 1.108683)
    skin = L0 / 5.01 - rc
    d = dict(d, pos=decks.fcc_reply_positions(12) * f + 0.2, box=(L0,) * 3, press_atm=1.0 * 1581225.25240563)
    s, rng_o = _oracle(d, skin=skin)
    s.interact()
    assert s.uses_cells() == (True, (5, 5, 5))
    E0, P0, V0 = decks.npt_run(s, d, rng_o, nsteps=100, each=20)
    assert s.uses_cells() == (True, (4, 4, 4)), "the compression did not change the oracle's grid"
    g = _gpu(ctx, d, skin=skin)
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(d["seed"]), nsteps=100, each=20, feed=_feed)
    np.testing.assert_allclose(g.box_now(), s.box_now(), rtol=1e-10)
    np.testing.assert_allclose(E1, E0, rtol=1e-8)
    np.testing.assert_allclose(V1, V0, rtol=1e-7, atol=1e-6)
    g.destroy()


def _gpu_axes(ctx, d, seed=12345, pos=None):
    g = gems.System(d["pos"] if pos is None else pos, d["mass"], ctx=ctx)
    g.set_skin_mode(False)
    decks.npt_axes_setup(g, d, seed)
    return g


@pytest.mark.parametrize("kind", ["flex", "x"])
def test_per_coordinate_decks(ctx, kind):
    """lgf_flex.gms (a piston on each length) and lgf_x.gms (a piston on x,
    Ermak on y and z) on the GPU with the LCG normals fed in draw order:
    the oracle's rows to 1e-9 and the golden files to their 7 digits."""
    d = decks.npt_axes_deck(kind)
    s = O.System(d["pos"], d["mass"])
    rng_o = O.Rng(d["seed"])
    decks.npt_axes_setup(s, d, rng_o)
    B0 = []
    E0, P0, V0 = decks.npt_run(s, d, rng_o, boxes=B0)
    g = _gpu_axes(ctx, d)
    B1 = []
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(d["seed"]), feed=_feed, boxes=B1)
    np.testing.assert_allclose(E1, E0, rtol=1e-9)
    np.testing.assert_allclose(P1, P0, rtol=1e-8, atol=1e-3)
    np.testing.assert_allclose(np.array(B1), np.array(B0), rtol=1e-12)
    E1[:, :3] *= O.UI_EV
    np.testing.assert_allclose(E1, d["ref_energy"], rtol=2e-6)
    np.testing.assert_allclose(P1, d["ref_press"], rtol=2e-6, atol=1e-2)
    if d["ref_virial"] is not None:
        np.testing.assert_allclose(V1, d["ref_virial"], rtol=2e-6, atol=1e-6)
    if d["ref_box"] is not None:
        np.testing.assert_allclose(np.array(B1), d["ref_box"], rtol=2e-7)
    g.destroy()


def test_per_coordinate_md_steps_and_resume(ctx):
    """lgf_flex with the device's own noise: the captured loop equals
    separate step calls bit for bit, and lgf_flex_a/b -- 60 steps,
    checkpoint, a fresh system restored from it, 60 more -- ends where the
    straight run does."""
    d = decks.npt_axes_deck("flex")
    a = _gpu_axes(ctx, d, seed=5)
    b = _gpu_axes(ctx, d, seed=5)
    a.interact()
    b.interact()
    a.md_steps(120)
    for _ in range(120):
        b.stepa()
        b.interact()
        b.stepb()
    np.testing.assert_array_equal(a.pos, b.pos)
    np.testing.assert_array_equal(a.vel, b.vel)
    np.testing.assert_array_equal(a.box_now(), b.box_now())
    L = a.box_now()
    assert abs(L[0] - L[1]) > 1e-4 and abs(L[0] - d["box"][0]) > 1e-3  # three independent lengths
    c = _gpu_axes(ctx, d, seed=5)
    c.md_steps(60)
    chp = c.checkpoint()
    c.destroy()
    e = _gpu_axes(ctx, d, seed=5, pos=np.zeros_like(d["pos"]))
    e.restore(chp)
    e.md_steps(60)
    np.testing.assert_allclose(e.box_now(), L, rtol=1e-10)
    np.testing.assert_allclose(e.pos, a.pos, rtol=0, atol=1e-8)
    for g in (a, b, e):
        g.destroy()


def test_lkd_trajectory_equals_oracle(ctx):
    """piston_lkd (no golden file in the reference): 100 steps with the
    oracle's normals fed in draw order, energies, pressure and box every
    10th step; then the captured loop against separate step calls."""
    d = decks.npt_lkd_deck()
    s, rng_o = _oracle(d)
    B0 = []
    E0, P0, V0 = decks.npt_run(s, d, rng_o, boxes=B0)
    g = gems.System(d["pos"], d["mass"], ctx=ctx)
    g.set_skin_mode(False)
    decks.npt_setup(g, d, 12345)
    B1 = []
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(d["seed"]), feed=_feed, boxes=B1)
    np.testing.assert_allclose(E1, E0, rtol=1e-9)
    np.testing.assert_allclose(P1, P0, rtol=1e-8, atol=1e-3)
    np.testing.assert_allclose(np.array(B1), np.array(B0), rtol=1e-12)
    assert abs(B1[-1][0] - d["box"][0]) > 1e-3
    g.destroy()
    a, b = [gems.System(d["pos"], d["mass"], ctx=ctx) for _ in range(2)]
    for x in (a, b):
        decks.npt_setup(x, d, 3)
        x.interact()
    a.md_steps(120)
    for _ in range(120):
        b.stepa()
        b.interact()
        b.stepb()
    np.testing.assert_array_equal(a.pos, b.pos)
    np.testing.assert_array_equal(a.box_now(), b.box_now())
    a.destroy()
    b.destroy()


# ------------------------------------------------------------------ GEMS .chp
_records = decks.chp_records


def test_gems_checkpoint_file_flex_split_run(ctx):
    """examples/test.sh's checkpoint case (lgf_flex_a.gms + lgf_flex_b.gms):
    50 steps, GEMS's checkpoint file, a fresh system resumed from it with the
    file's LCG state, 50 more; the concatenated energies are
    Energy.lgf_flex.dat.  The file is checked record by record against the
    layout of write_chp and the oracle's piston state after 50 steps."""
    import struct
    d = decks.npt_axes_deck("flex")
    n = len(d["pos"])
    g = _gpu_axes(ctx, d)
    rng = O.Rng(d["seed"])
    Ea, Pa, Va = decks.npt_run(g, d, rng, nsteps=50, feed=_feed)
    state = rng.chp_state()
    chp = g.write_gems_chp(current=1, step=50, nsteps=50, rng=state, time=50 * d["dt"], frame=5)
    r = _records(chp)
    assert struct.unpack("<4i", r[0]) == (1, 50, 50, n)
    tbox = np.array(struct.unpack("<9d", r[1])).reshape(3, 3, order="F")
    np.testing.assert_array_equal(np.diag(tbox), g.box_now())
    assert r[2] == b"lcg" and struct.unpack("<3i", r[3]) == state
    assert struct.unpack("<3i", r[4]) == (1, 1, 1)
    s, rng_o = O.System(d["pos"], d["mass"]), O.Rng(d["seed"])
    decks.npt_axes_setup(s, d, rng_o)
    decks.npt_run(s, d, rng_o, nsteps=50)
    pf, pv = s.piston_state()
    for k in range(3):
        ppos, pvel, pistonf = (struct.unpack("<d", r[5 + 3 * k + q])[0] for q in range(3))
        assert ppos == 0.0
        assert abs(pvel - pv[k]) <= 1e-9 * abs(pv[k]) and abs(pistonf - pf[k]) <= 1e-9 * abs(pf[k])
    fr = struct.unpack("<5di", r[14])
    assert fr[1] == 50 * d["dt"] and fr[5] == 5
    atoms = r[15:]
    assert len(atoms) == 6 * n
    np.testing.assert_array_equal(np.array([struct.unpack("<3d", atoms[6 * i]) for i in range(n)]), g.pos)
    g.destroy()
    h = _gpu_axes(ctx, d, pos=np.zeros_like(d["pos"]))
    info = h.read_gems_chp(chp)
    assert info["step"] == 50 and info["rng"] == state and info["frame"] == 5
    rng_b = O.Rng(1)
    rng_b.set_state(*info["rng"])
    Eb, Pb, Vb = decks.npt_run(h, d, rng_b, nsteps=50, feed=_feed)
    E = np.vstack([Ea, Eb])
    E[:, :3] *= O.UI_EV
    np.testing.assert_allclose(E, d["ref_energy"], rtol=2e-6)
    np.testing.assert_allclose(np.vstack([Pa, Pb]), d["ref_press"], rtol=2e-6, atol=1e-2)
    h.destroy()


def test_gems_checkpoint_file_from_gems(ctx):
    """A file laid out as GEMS writes it (an 'std' generator record, no
    piston) resumes an NVT system: positions, velocities, accelerations,
    the box and the counters; a wrong atom count and a cut file are errors."""
    import struct
    d = decks.npt_lgf_deck()
    n = len(d["pos"])
    rng = np.random.default_rng(4)
    x = np.mod(d["pos"] + rng.normal(0, 0.05, d["pos"].shape), d["box"][0] * 0.999)
    v = rng.normal(0, 1.0, x.shape)
    a = rng.normal(0, 1.0, x.shape)
    L = np.array(d["box"]) * 0.999

    def rec(b):
        return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    data = rec(struct.pack("<4i", 3, 700, 1000, n)) + rec(np.diag(L).flatten(order="F").tobytes())
    data += rec(b"std") + rec(struct.pack("<i", 2)) + rec(struct.pack("<2i", 11, 12))
    data += rec(struct.pack("<3i", 0, 0, 0)) + rec(struct.pack("<5di", 7.0, 1.4, 700.0, 0.0, 0.0, 7))
    for i in range(n):
        for arr in (x[i], v[i], a[i], np.zeros(3), np.zeros(3), np.zeros(3)):
            data += rec(np.asarray(arr, dtype="<f8").tobytes())
    g = gems.System(np.zeros_like(x), d["mass"], ctx=ctx)
    g.set_box(d["box"], (True, True, True))
    g.set_slj(*d["slj"])
    g.set_ermak(d["dt"], 10.0, 300.0)
    info = g.read_gems_chp(data)
    assert (info["current"], info["step"], info["nsteps"], info["frame"]) == (3, 700, 1000, 7)
    np.testing.assert_array_equal(g.pos, x)
    np.testing.assert_array_equal(g.vel, v)
    np.testing.assert_array_equal(g.acel, a)
    np.testing.assert_array_equal(g.box_now(), L)
    g.interact()
    g.md_steps(5)
    for bad in (data[:-10], data[:40]):
        with pytest.raises(gems.GemsGpuError):
            g.read_gems_chp(bad)
    small = gems.System(x[:10], d["mass"], ctx=ctx)
    small.set_box(d["box"], (True, True, True))
    with pytest.raises(gems.GemsGpuError):
        small.read_gems_chp(data)
    g.destroy()
    small.destroy()


def test_smatb_virial_and_piston_equal_oracle(ctx):
    """The pistons on a metal: the SMA-TB force pass sums the pair virial
    (the complete sum of the central pair forces), and an Au crystal under
    the isotropic G-JF piston at 1 atm follows the oracle for 100 steps with
    the oracle's normals fed to the device."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)
    rng = np.random.default_rng(9)
    pos = np.mod(w["pos"] + rng.normal(0, 0.05, w["pos"].shape), w["L"])
    s = O.System(pos, w["mass"])
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    g = gems.System(pos, w["mass"], ctx=ctx)
    g.set_skin_mode(False)
    g.set_box(w["L"], (True, True, True))
    g.set_smatb(*w["smatb"])
    g.set_virial(True)
    s.interact()
    g.interact()
    np.testing.assert_allclose(g.virial_ev(), s.virial_ev(), rtol=1e-10, atol=1e-8)
    d = dict(dt=w["dt"], nsteps=100, each=10)
    s.set_lgf(w["dt"], 300.0, 1.0, 1.0, 1.0, 1e-3, O.Rng(7))
    g.set_lgf(w["dt"], 300.0, 1.0, 1.0, 1.0, 1e-3)
    rng_o = s._rng
    B0, B1 = [], []
    E0, P0, V0 = decks.npt_run(s, d, rng_o, boxes=B0)
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(7), feed=_feed, boxes=B1)
    np.testing.assert_allclose(E1, E0, rtol=1e-9)
    np.testing.assert_allclose(V1, V0, rtol=1e-8, atol=1e-6)
    np.testing.assert_allclose(np.array(B1), np.array(B0), rtol=1e-12)
    assert abs(B1[-1][0] - w["L"][0]) > 1e-4
    g.destroy()


@pytest.mark.parametrize("ff", ["smatb", "lj"])
def test_mixed_precision_virial(ctx, ff):
    """Mixed precision sums the pair virial in FP32 per pair and FP64 per
    atom and system; its tensor matches the oracle's within the mixed
    kernels' force tolerance (1e-5 of its largest component)."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)
    rng = np.random.default_rng(12)
    pos = np.mod(w["pos"] + rng.normal(0, 0.05, w["pos"].shape), w["L"])
    s = O.System(pos, w["mass"])
    g = gems.System(pos, w["mass"], ctx=ctx)
    for x in (s, g):
        x.set_box(w["L"], (True, True, True))
        if ff == "smatb":
            x.set_smatb(*w["smatb"])
        else:
            x.set_lj(0.2, 2.6, 6.0, shifted_force=True)
    g.set_precision(1)
    g.set_virial(True)
    s.interact()
    g.interact()
    ref = s.virial_ev()
    np.testing.assert_allclose(g.virial_ev(), ref, rtol=0, atol=1e-5 * np.abs(ref).max())
    p = g.pressure_atm()
    assert np.all(np.isfinite(p))
    g.destroy()


# Mixed precision under the pistons: the fixed-point frame of the mixed kernels
# follows the box the device moves, so the constant-pressure integrators run
# the FP32-math / FP64-accumulation kernels.  Measured against the oracle's
# FP64 rows over these runs: energies within 3.1e-7 eV/atom, pressure and
# virial within 5e-6 of their largest component, box lengths within 1.5e-7 A.
E_MIXED = 1e-6        # eV per atom (the mixed kernels' energy bar)
P_MIXED = 2e-5        # of the largest pressure / virial component
BOX_MIXED = 1e-6      # relative box length


def _mixed_rows_close(n, E1, P1, V1, E0, P0, V0):
    assert np.abs(E1[:, :3] - E0[:, :3]).max() * O.UI_EV / n <= E_MIXED
    assert np.abs(P1 - P0).max() <= P_MIXED * np.abs(P0).max()
    assert np.abs(V1 - V0).max() <= P_MIXED * np.abs(V0).max()


def test_lgf_deck_mixed_precision(ctx):
    """lgf.gms (864 slj atoms, isotropic G-JF piston, 100 steps) in mixed
    precision, the oracle's normals fed in, against the oracle's FP64 rows."""
    d = decks.npt_lgf_deck()
    s, rng_o = _oracle(d)
    E0, P0, V0 = decks.npt_run(s, d, rng_o)
    g = _gpu(ctx, d)
    g.set_precision(1)
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(d["seed"]), feed=_feed)
    _mixed_rows_close(len(d["pos"]), E1, P1, V1, E0, P0, V0)
    np.testing.assert_allclose(g.box_now(), s.box_now(), rtol=BOX_MIXED)
    g.destroy()


def test_smatb_piston_mixed_precision(ctx):
    """An Au crystal (864 atoms) under the isotropic G-JF piston at 1 atm,
    100 steps in mixed precision, against the oracle's FP64 rows and boxes."""
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)
    rng = np.random.default_rng(9)
    pos = np.mod(w["pos"] + rng.normal(0, 0.05, w["pos"].shape), w["L"])
    s = O.System(pos, w["mass"])
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    g = gems.System(pos, w["mass"], ctx=ctx)
    g.set_skin_mode(False)
    g.set_box(w["L"], (True, True, True))
    g.set_smatb(*w["smatb"])
    g.set_virial(True)
    g.set_precision(1)
    d = dict(dt=w["dt"], nsteps=100, each=10)
    s.set_lgf(w["dt"], 300.0, 1.0, 1.0, 1.0, 1e-3, O.Rng(7))
    g.set_lgf(w["dt"], 300.0, 1.0, 1.0, 1.0, 1e-3)
    B0, B1 = [], []
    E0, P0, V0 = decks.npt_run(s, d, s._rng, boxes=B0)
    E1, P1, V1 = decks.npt_run(g, d, O.Rng(7), feed=_feed, boxes=B1)
    _mixed_rows_close(len(pos), E1, P1, V1, E0, P0, V0)
    np.testing.assert_allclose(np.array(B1), np.array(B0), rtol=BOX_MIXED)
    assert abs(B1[-1][0] - w["L"][0]) > 1e-4      # the box did move
    g.destroy()
