"""L-BFGS on the GPU (lbfgs_minimizator, src/Quasi_Newton.f90) against the
oracle, the examples/SMA-TB/md.gms golden file, and itself in a batch."""
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


def test_md_deck_lbfgs_then_ermak(ctx):
    """md.gms end to end on the GPU: L-BFGS of 13 Ag to the oracle's minimum,
    then 1000 Ermak steps on the LCG stream against Energy.md.dat."""
    d = decks.md_deck()
    o = O.System(d["pos"], d["mass"])
    o.set_smatb(*d["smatb"])
    oflag, _, _, oe = o.lbfgs()
    assert oflag == 0
    g = gems.System(d["pos"], d["mass"], ctx=ctx)
    g.set_skin_mode(False)
    g.set_smatb(*d["smatb"])
    st, it, nf, e = g.lbfgs()
    assert st == 0 and nf < 100
    assert abs(e - oe) < 1e-9
    np.testing.assert_allclose(g.pos, o.pos, atol=1e-6)
    g.set_ermak(d["dt"], d["gamma"], d["temp"])
    rows = decks.ermak_parity_run(g, O.Rng(d["seed"]), d["nsteps"], d["each"])
    got = rows[:, :3] * gems.UI_EV
    assert decks.gems_rule(d["ref"][:, 0], got[:, 0]) < 1e-6
    np.testing.assert_allclose(got, d["ref"], rtol=1e-6, atol=1e-6)
    g.destroy()


def _clusters():
    """Jittered cluster cuts placed about (200, 200, 200) A, where GEMS decks
    put them (md.gms): the stopping rule |g| <= eps int(max(1, |x|)) scales
    with |x|, and at the origin it would ask for a gradient below what FP64
    resolves in f."""
    from gems_b200 import workloads as W
    return [W.cluster(n, np.random.default_rng(100 + n), jitter=0.15) + 200.0 for n in (13, 38, 147, 309)]


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_lbfgs_equals_alone_and_reaches_oracle_minimum(ctx, prec):
    from gems_b200 import workloads as W
    sm, m = W.SMATB["Au"], W.MASS["Au"]
    cl = _clusters()

    def mk(p):
        g = gems.System(p, m, ctx=ctx)
        g.set_smatb(*sm)
        g.set_precision(prec)
        g.set_lanes(4, 1)
        return g

    alone = []
    for p in cl:
        g = mk(p)
        alone.append((g.lbfgs(), g.pos))
        g.destroy()
    batch = [mk(p) for p in cl]
    st, it, nf, em = ctx.batch_lbfgs(batch)
    for k, (g, p) in enumerate(zip(batch, cl)):
        (st1, it1, nf1, e1), pos1 = alone[k]
        assert (st[k], it[k], nf[k], em[k]) == (st1, it1, nf1, e1)   # bit for bit
        np.testing.assert_array_equal(g.pos, pos1)
        o = O.System(p, m)
        o.set_smatb(*sm)
        oflag, _, _, oe = o.lbfgs()
        assert oflag in (0, -1)
        if prec == 0:
            assert st[k] in (0, -1)
            assert abs(em[k] - oe) / len(p) < 1e-9
        else:
            # FP32 pair math: the search ends converged or when the line
            # search can no longer resolve the noise of f near the minimum
            assert st[k] in (0, -1)
            assert abs(em[k] - oe) / len(p) < 2e-6
        assert g.fmax() < 2e-3
    for g in batch:
        g.destroy()
