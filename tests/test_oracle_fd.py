"""The oracle's forces are minus the gradient of its energy (CPU only).

Tersoff and FIRE have no golden file in the reference, so the Tersoff
restatement is pinned here by central finite differences; LJ and SMA-TB are
checked the same way for completeness.
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
