"""Nudged elastic band on the GPU (neb, src/NEB.f90) against the oracle and
the examples/NEB/neb.gms golden file."""
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


def _gpu_system(ctx, d, pos):
    g = gems.System(pos, d["mass"], d["types"], 2, ctx=ctx)
    decks.neb_setup(g, d)
    return g


def _oracle_fixed_images(d):
    s = O.System(d["pos"], d["mass"], d["types"], 2)
    decks.neb_setup(s, d)
    return s, decks.neb_fixed_images(s, d, lambda x: x.lbfgs())


def test_neb_band_equals_oracle(ctx):
    """Same fixed images in, the same band out: 30 images, 20 iterations."""
    d = decks.neb_deck()
    s, imgs = _oracle_fixed_images(d)
    ref_band, ref_dt = s.neb(imgs, d["fixed"], d["k"], d["iters"])
    images = [_gpu_system(ctx, d, imgs[k]) for k in range(d["nimg"])]
    dt, e = ctx.neb(images, d["fixed"], d["k"], d["iters"])
    assert abs(dt - ref_dt) / ref_dt < 1e-12
    band = np.array([g.pos for g in images])
    np.testing.assert_allclose(band, ref_band, rtol=0, atol=1e-8)
    for k in (0, 7, 14, 29):
        s.set_pos(ref_band[k])
        s.interact()
        assert abs(e[k] - s.epot_sum() * O.UI_EV) < 1e-8
    for g in images:
        g.destroy()


def test_neb_deck_end_to_end(ctx):
    """neb.gms on the GPU: the three fixed images relaxed by the device
    L-BFGS, then the band, against Energy.neb.dat.NebF by the reference's
    rule for this deck (test.sh: < 1e-4)."""
    d = decks.neb_deck()
    g = _gpu_system(ctx, d, d["pos"])
    imgs = decks.neb_fixed_images(g, d, lambda x: x.lbfgs())
    g.destroy()
    images = [_gpu_system(ctx, d, imgs[k]) for k in range(d["nimg"])]
    dt, e = ctx.neb(images, d["fixed"], d["k"], d["iters"])
    band = np.array([x.pos for x in images])
    rows = decks.neb_rows(band, e)
    assert decks.neb_rule(d["ref"], rows) < 1e-4
    np.testing.assert_allclose(rows[:, 0], d["ref"][:, 0], atol=1e-5)
    np.testing.assert_allclose(rows[:, 1], d["ref"][:, 1], atol=1e-2)
    for x in images:
        x.destroy()
