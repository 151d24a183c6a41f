"""Checkpoint/resume and NVE energy drift on the GPU.

* examples/NVT/ermak_a.gms + ermak_b.gms: 5000 Ermak steps, checkpoint, a
  fresh system restored from it, 5000 more steps; the concatenated energies
  must reproduce ref/Energy.ermak.dat (the rule of examples/test.sh).
* NVE drift over 10^4 steps: the GPU's (FP64 and mixed) total-energy drift
  stays within the oracle's for the LJ fluid and the Tersoff crystal.
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


def _drift(etot, n):
    """Largest excursion of the total energy from its first row, eV/atom."""
    return float(np.max(np.abs(etot - etot[0]))) / n


def test_nve_drift_lj(ctx):
    """864-atom LJ fluid (rho*=0.8442, T*=0.72, shifted-force), 10^4 VV steps."""
    from gems_b200 import workloads as W
    rho = 0.8442
    a = (4.0 / rho) ** (1.0 / 3.0)
    pos = W.fcc(6, a)
    L = 6 * a
    vel = W.maxwell(len(pos), 1.0, 0.72 / W.KB_EV, np.random.default_rng(7))
    dt = 0.005 * np.sqrt(W.UI_EV)

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_lj(1.0, 1.0, 2.5, shifted_force=True)
        s.set_skin(0.3)
        s.set_vv(dt)

    o = O.System(pos, 1.0)
    o.set_vel(vel)
    setup(o)
    drift_o = _drift(o.dinamica(10000, 500)[:, 2], len(pos))
    for prec in (gems.PREC_FP64, gems.PREC_MIXED):
        g = gems.System(pos, 1.0, ctx=ctx, vel=vel)
        setup(g)
        g.set_precision(prec)
        drift_g = _drift(g.dinamica(10000, 500)[:, 2], len(pos))
        assert drift_g <= 2.0 * drift_o + 1e-6, (prec, drift_g, drift_o)


def test_nve_drift_tersoff(ctx):
    """512-atom Tersoff Si(C) diamond at 1000 K, 10^4 VV steps of 1 fs."""
    from gems_b200 import workloads as W
    pos = W.diamond(4, 5.431)
    L = 4 * 5.431
    vel = W.maxwell(len(pos), W.MASS["Si"], 1000.0, np.random.default_rng(5))

    def setup(s):
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
        s.set_vv(0.001)

    o = O.System(pos, W.MASS["Si"])
    o.set_vel(vel)
    setup(o)
    drift_o = _drift(o.dinamica(10000, 500)[:, 2], len(pos))
    for prec in (gems.PREC_FP64, gems.PREC_MIXED):
        g = gems.System(pos, W.MASS["Si"], ctx=ctx, vel=vel)
        setup(g)
        g.set_precision(prec)
        drift_g = _drift(g.dinamica(10000, 500)[:, 2], len(pos))
        assert drift_g <= 2.0 * drift_o + 1e-6, (prec, drift_g, drift_o)
