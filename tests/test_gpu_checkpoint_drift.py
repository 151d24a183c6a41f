"""Checkpoint/resume and NVE energy drift on the GPU.

* examples/NVT/ermak_a.gms + ermak_b.gms: 5000 Ermak steps, checkpoint, a
  fresh system restored from it, 5000 more steps; the concatenated energies
  must reproduce ref/Energy.ermak.dat (the rule of examples/test.sh).
* NVE drift over 10^4 steps: the GPU's (FP64 and mixed) total-energy drift
  stays within the oracle's on the C1 LJ fluid itself and on a 4096-atom
  Tersoff crystal.
"""
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


def _ermak_rows(g, rng, nsteps, each, first=True):
    if first:
        g.interact()
    rows = []
    for ns in range(1, nsteps + 1):
        g.set_ermak_normals(rng.rang_stream(3 * g.n))
        g.stepa()
        g.interact()
        g.stepb()
        if ns % each == 0:
            ep, ek, t = g.energy()
            rows.append([ep, ek, ep + ek, t])
    return rows


def test_nvt_checkpoint_split_run(ctx):
    pos, vel, types, mass, box, rng = decks.he_ne_setup(O)

    def mk(p, v):
        g = gems.System(p, mass, types, 2, ctx=ctx, vel=v)
        g.set_skin_mode(False)
        g.set_box(box, (True, True, True))
        decks.apply_plj(g)
        g.set_ermak(0.002, 10.0, 300.0)
        return g

    a = mk(pos, vel)
    rows = _ermak_rows(a, rng, 5000, 100)
    chp = a.checkpoint()
    a.destroy()
    b = mk(np.zeros_like(pos), None)       # a fresh system: everything comes from the checkpoint
    b.restore(chp)
    rows += _ermak_rows(b, rng, 5000, 100)
    ref = np.array(decks.golden()["nvt_energy"])
    rows = np.array(rows)
    assert decks.gems_rule(ref[:, 0], rows[:, 0]) < 1e-6
    np.testing.assert_allclose(rows[:, 3], ref[:, 3], rtol=1e-5)


def test_checkpoint_roundtrip_state(ctx):
    from gems_b200 import workloads as W
    w = W.smatb_bulk(ncell=6)
    g = gems.System(w["pos"], w["mass"], ctx=ctx)
    g.set_box(w["L"], (True, True, True))
    g.set_smatb(*w["smatb"])
    g.set_ermak(0.002, 1.0, 300.0, seed=5)
    g.interact()
    g.md_steps(150)
    chp = g.checkpoint()
    p0, v0, a0 = g.pos, g.vel, g.acel
    g.md_steps(100)
    e_cont = g.energy()
    g.restore(chp)
    np.testing.assert_array_equal(g.pos, p0)
    np.testing.assert_array_equal(g.vel, v0)
    np.testing.assert_array_equal(g.acel, a0)
    g.md_steps(100)                         # same Philox counters: same dynamics
    e_res = g.energy()
    assert abs(e_res[0] - e_cont[0]) / abs(e_cont[0]) < 1e-9


def _drift(e):
    """Largest excursion of the total energy per atom from its first row."""
    return float(np.max(np.abs(e - e[0])))


def _rows(s, nsteps, each, n):
    return s.dinamica(nsteps, each)[:, 2] / n


def test_nve_drift_c1_lj(ctx):
    """The C1 workload itself: 4000 atoms on an fcc 10^3 lattice at
    rho* = 0.8442, Maxwell-Boltzmann velocities at T* = 0.72 (seed 1, zero
    momentum), truncated-and-shifted LJ (rc = 2.5 sigma, lj with the energy
    shift), skin 0.3 sigma, 10^4 velocity-Verlet steps of 0.005 tau, a row
    every 10 steps.

    Drift = the largest |E(t) - E(first row)| per atom.  From the lattice
    start it is set by the transient as the crystal melts, not by the seed:
    the oracle's seeds 1-4 give 7.13e-4 .. 7.61e-4 eV/atom (max/min 1.07),
    and the GPU's drift on the same seed has matched the oracle's to 0.1 %.
    The GPU's drift (FP64 and mixed) must stay within the oracle's on the
    same seed; the 1 % allowance is a seventh of the oracle's own spread over
    seeds.  Before chaos separates the trajectories the rows themselves must
    agree: FP64 over the first 1000 steps to 1e-10 eV/atom, mixed over the
    first 200 steps to 1e-6 eV/atom."""
    from gems_b200 import workloads as W
    w = W.lj_fluid(seed=1)
    n = len(w["pos"])

    def setup(s):
        s.set_box(w["L"], (True, True, True))
        e, sg, rc, sh = w["lj"]
        s.set_lj(e, sg, rc, eshift=sh)
        s.set_skin(w["skin"])
        s.set_skin_mode(True)
        s.set_vv(w["dt"])

    o = O.System(w["pos"], 1.0)
    o.set_vel(w["vel"])
    setup(o)
    eo = _rows(o, 10000, 10, n)
    drift_o = _drift(eo)
    for prec, nrows, tol in ((gems.PREC_FP64, 100, 1e-10), (gems.PREC_MIXED, 20, 1e-6)):
        g = gems.System(w["pos"], 1.0, ctx=ctx, vel=w["vel"])
        setup(g)
        g.set_precision(prec)
        eg = _rows(g, 10000, 10, n)
        assert np.abs(eg[:nrows] - eo[:nrows]).max() <= tol, (prec, np.abs(eg[:nrows] - eo[:nrows]).max())
        drift_g = _drift(eg)
        assert drift_g <= 1.01 * drift_o, (prec, drift_g, drift_o)
        g.destroy()


def test_nve_drift_tersoff(ctx):
    """4096-atom Tersoff Si(C) diamond (8^3 cells) with Maxwell-Boltzmann
    velocities at 1000 K (seed 5), 10^4 velocity-Verlet steps of 1 fs, a row
    every 20 steps.  The drift (largest |E(t) - E(first row)| per atom) is the
    systematic level shift of the lattice start: the oracle's seeds 5 and 6
    give 8.88e-5 and 9.01e-5 eV/atom.  The GPU's (FP64 and mixed) must stay
    within 1 % of the oracle's on the same seed."""
    from gems_b200 import workloads as W
    pos = W.diamond(8, 5.431)
    L = 8 * 5.431
    vel = W.maxwell(len(pos), W.MASS["Si"], 1000.0, np.random.default_rng(5))

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
        s.set_skin_mode(True)
        s.set_vv(0.001)

    o = O.System(pos, W.MASS["Si"])
    o.set_vel(vel)
    setup(o)
    drift_o = _drift(_rows(o, 10000, 20, len(pos)))
    for prec in (gems.PREC_FP64, gems.PREC_MIXED):
        g = gems.System(pos, W.MASS["Si"], ctx=ctx, vel=vel)
        setup(g)
        g.set_precision(prec)
        drift_g = _drift(_rows(g, 10000, 20, len(pos)))
        assert drift_g <= 1.01 * drift_o, (prec, drift_g, drift_o)
        g.destroy()
