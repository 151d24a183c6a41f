"""The oracle's forces are minus the gradient of its energy (CPU only).

Tersoff and FIRE have no golden file in the reference, so the Tersoff
restatement is pinned here by central finite differences; LJ, WCA and SMA-TB
are checked the same way for completeness.  Two pair forms are deliberately
not gradients, as in the reference: sm1's force carries a factor r, and a
one-sided (feels) pair puts the whole force on one atom while counting half
the energy.
"""
import numpy as np
import pytest

from oracle import oracle as O


def fd_check(make, pos, atoms, h=1e-5, rtol=2e-6):
    s = make(pos)
    s.interact()
    f = s.force
    for i in atoms:
        for k in range(3):
            ep = []
            for sgn in (1, -1):
                p = pos.copy()
                p[i, k] += sgn * h
                t = make(p)
                ep.append(t.interact())
            num = -(ep[0] - ep[1]) / (2 * h)
            assert abs(num - f[i, k]) <= rtol * max(1.0, np.abs(f).max()), (i, k, num, f[i, k])


def test_tersoff_fd():
    from gems_b200 import workloads as W
    rng = np.random.default_rng(4)
    L = 3 * 5.431
    pos = np.mod(W.diamond(3, 5.431) + rng.normal(0, 0.08, (216, 3)), L)

    def make(p):
        s = O.System(p, W.MASS["Si"])
        s.set_box((L, L, L), (True, True, True))
        s.set_tersoff(W.TERSOFF_SI)
        return s

    fd_check(make, pos, atoms=[0, 5, 77])


def test_tersoff_cutoff_region_fd():
    """Bonds inside the smooth cut-off (R-D < r < R+D) and angles near h."""
    from gems_b200 import workloads as W
    pos = np.array([[0.0, 0, 0], [2.2, 0.3, 0], [-1.1, 2.0, 0.2], [0.4, -0.6, 2.86],
                    [-2.75, -0.4, -0.3]])

    def make(p):
        s = O.System(p, W.MASS["Si"])
        s.set_tersoff(W.TERSOFF_SI)
        return s

    fd_check(make, pos, atoms=range(5))


@pytest.mark.parametrize("element", ["Au", "Ag"])
def test_smatb_fd(element):
    from gems_b200 import workloads as W
    pos = W.cluster(60, np.random.default_rng(1))

    def make(p):
        s = O.System(p, W.MASS[element])
        s.set_smatb(*W.SMATB[element])
        return s

    fd_check(make, pos, atoms=[0, 30, 59])


def test_lj_shifted_force_fd():
    rng = np.random.default_rng(2)
    pos = rng.uniform(0, 12, (40, 3))
    pos = pos[np.argsort(pos[:, 0])]

    def make(p):
        s = O.System(p, 4.0)
        s.set_box((12.0, 12.0, 12.0), (True, True, True))
        s.set_lj(0.01, 2.0, 5.0, shifted_force=True)
        return s

    fd_check(make, pos, atoms=[0, 20])


def test_wca_fd():
    """wca: a compressed periodic fluid, every pair force the exact gradient."""
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 6, (60, 3))

    def make(p):
        s = O.System(p, 4.0)
        s.set_box((6.0, 6.0, 6.0), (True, True, True))
        s.set_wca(0.01, 1.3)
        return s

    fd_check(make, pos, atoms=[0, 31])


def _dimer(p, setup, types=(0, 0), ntypes=1):
    s = O.System(p, 4.0, np.array(types), ntypes)
    setup(s)
    return s


def _grad(setup, pos, i, k, h=1e-6, **kw):
    ep = []
    for sgn in (1, -1):
        p = pos.copy()
        p[i, k] += sgn * h
        ep.append(_dimer(p, setup, **kw).interact())
    return (ep[0] - ep[1]) / (2 * h)


@pytest.mark.parametrize("r", [1.2, 1.5, 1.93])
def test_sm1_force_is_r_times_gradient(r):
    """sm1 keeps the reference's force, f = r dp/dr (src/Pairs.F90:957):
    between r1 and r2 the oracle's force is r times minus the gradient."""
    pos = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])

    def setup(s):
        s.set_sm1(1.0, 2.0, 0.5)

    s = _dimer(pos, setup)
    s.interact()
    f = s.force
    g = _grad(setup, pos, 0, 0)
    assert abs(f[0, 0] - r * (-g)) <= 1e-6 * abs(f[0, 0])
    assert abs(f[1, 0] + f[0, 0]) <= 1e-12 * abs(f[0, 0])


def test_feels_is_one_sided():
    """`feels`: the feeling atom takes the whole pair force, the other none;
    the energy counts the feeling side's half, so that force is minus twice
    the gradient of the reported energy."""
    pos = np.array([[0.0, 0.0, 0.0], [1.05, 0.2, -0.1]])

    def setup(s):
        s.set_wca(1.0, 1.0, ti=1, tj=0)
        s.set_feels(1, 0)

    s = _dimer(pos, setup, types=(0, 1), ntypes=2)
    e = s.interact()
    f = s.force
    assert np.all(f[0] == 0.0) and np.abs(f[1]).max() > 0.0
    full = _dimer(pos, lambda t: t.set_wca(1.0, 1.0, ti=1, tj=0), types=(0, 1), ntypes=2)
    assert abs(2 * e - full.interact()) <= 1e-12 * abs(e)
    for k in range(3):
        g = _grad(setup, pos, 1, k, types=(0, 1), ntypes=2)
        assert abs(f[1, k] + 2 * g) <= 1e-6 * np.abs(f[1]).max()
