"""Synthetic, seeded inputs of the benchmark configurations.

The reference ships no benchmark inputs, so each configuration is generated
here from its definition: lattice, box, species parameters, displacement or
velocity distribution and seed.  Numbers in internal GEMS units (Angstrom,
uma, ps) unless noted.
"""
import math

import numpy as np

# element masses (src/Elements.F90, single-precision literals widened)
MASS = {"Ag": float(np.float32(107.87)), "Au": float(np.float32(196.97)),
        "Pt": float(np.float32(195.08)), "Si": float(np.float32(28.09))}

# SMA-TB (Cleri & Rosato 1993 A, xi, p, q, r0); Au cut-offs rci=4.4, rce=5.0,
# Ag/Pt cut-offs scaled by r0 with the Au ratio
SMATB = {
    "Au": (0.2061, 1.790, 10.229, 4.036, 2.884, 4.4, 5.0),
    "Ag": (0.1028, 1.178, 10.928, 3.139, 2.889, 2.889 * 4.4 / 2.884, 2.889 * 5.0 / 2.884),
    "Pt": (0.2975, 2.695, 10.612, 4.004, 2.775, 2.775 * 4.4 / 2.884, 2.775 * 5.0 / 2.884),
}

# Tersoff Si(C) (Tersoff 1988): A, B (eV), lambda1, lambda2, beta, n, c, d, h, R, D, chi
TERSOFF_SI = (1830.8, 471.18, 2.4799, 1.7322, 1.1e-6, 0.78734, 100390.0, 16.217, -0.59825,
              2.85, 0.15, 1.0)

KB_EV = 8.617385e-05
UI_EV = 1.0e2 * 1.0e2 * 1.6605402e-27 * (1.0 / 1.60219e-19)
EV_UI = 1.0 / UI_EV
KB_UI = KB_EV * EV_UI


def fcc(ncell, a):
    """fcc lattice of ncell^3 cubic cells (4 atoms each), cell-major order."""
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)
    g = np.arange(ncell, dtype=np.float64)
    cz, cy, cx = np.meshgrid(g, g, g, indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    pos = (cells[:, None, :] + base[None, :, :]).reshape(-1, 3) * a
    return pos


def diamond(ncell, a):
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5],
                     [0.25, 0.25, 0.25], [0.75, 0.75, 0.25], [0.75, 0.25, 0.75],
                     [0.25, 0.75, 0.75]], dtype=np.float64)
    g = np.arange(ncell, dtype=np.float64)
    cz, cy, cx = np.meshgrid(g, g, g, indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    return (cells[:, None, :] + base[None, :, :]).reshape(-1, 3) * a


def maxwell(n, mass, temp, rng):
    """Maxwell-Boltzmann velocities at temp (K), zero net momentum, rescaled
    to exactly temp (the set_gdist recipe, src/Set_Properties.f90:301-349)."""
    m = np.broadcast_to(np.asarray(mass, dtype=np.float64), (n,))
    v = rng.standard_normal((n, 3)) * np.sqrt(KB_UI * temp / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    ek = 0.5 * (m[:, None] * v * v).sum()
    t = 2.0 * ek / (KB_UI * 3 * n)
    if t > 0:
        v *= math.sqrt(temp / t)
    return v


def lj_fluid(seed=1):
    """C1: 4000 LJ atoms, fcc 10^3 at rho*=0.8442, T*=0.72, rc=2.5, skin 0.3."""
    rho = 0.8442
    a = (4.0 / rho) ** (1.0 / 3.0)
    pos = fcc(10, a)
    L = 10 * a
    rng = np.random.default_rng(seed)
    T = 0.72 / KB_EV              # eps = 1 eV, so T* = kB T / eps
    vel = maxwell(len(pos), 1.0, T, rng)
    rc = 2.5
    eshift = 4.0 * ((1.0 / rc) ** 12 - (1.0 / rc) ** 6)   # eV, truncated and shifted
    tau = math.sqrt(UI_EV)         # ps, for sigma = 1 A, m = 1 uma, eps = 1 eV
    return dict(name="lj_fluid_4000", pos=pos, vel=vel, mass=1.0, L=(L, L, L), pbc=(1, 1, 1),
                lj=(1.0, 1.0, rc, eshift), skin=0.3, dt=0.005 * tau, nsteps=1000)


def smatb_bulk(seed=2, ncell=20, element="Au"):
    """C2: 32000-atom Au fcc 20^3 (a=4.078), sigma=0.02 A displacements,
    Ermak 300 K, gamma=1/ps, dt=2 fs."""
    a = 4.078
    pos = fcc(ncell, a)
    L = ncell * a
    rng = np.random.default_rng(seed)
    pos = pos + rng.normal(0.0, 0.02, pos.shape)
    pos = np.mod(pos, L)
    return dict(name="smatb_au_bulk_%d" % len(pos), pos=pos, mass=MASS[element], L=(L, L, L),
                pbc=(1, 1, 1), smatb=SMATB[element], skin=1.0, dt=0.002, temp=300.0, gamma=1.0,
                nsteps=5000)


def tersoff_si(seed=5, ncell=50):
    """C5: diamond Si 50^3 (1,000,000 atoms), a=5.431, MB 1000 K, VV dt=1 fs."""
    a = 5.431
    pos = diamond(ncell, a)
    L = ncell * a
    rng = np.random.default_rng(seed)
    vel = maxwell(len(pos), MASS["Si"], 1000.0, rng)
    return dict(name="tersoff_si_%d" % len(pos), pos=pos, vel=vel, mass=MASS["Si"], L=(L, L, L),
                pbc=(1, 1, 1), tersoff=TERSOFF_SI, skin=1.0, dt=0.001, nsteps=2000)


def cluster(n, rng, dmin=2.5, a=4.078, jitter=0.05, check=True):
    """A compact n-atom blob at bulk fcc density: the n sites of a randomly
    rotated and shifted fcc lattice (lattice constant a) nearest to the
    centre, each displaced by N(0, jitter); every pair stays >= dmin apart.
    (Random sequential addition, the create_fill rule of
    src/Select_Create.F90:64-135, jams below bulk density at dmin=2.5 A.)"""
    if n <= 0:
        return np.zeros((0, 3))
    m = int(math.ceil((n / 4.0) ** (1.0 / 3.0))) + 3
    pos = fcc(2 * m, a) - m * a
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    pos = pos @ q.T + rng.uniform(-0.5, 0.5, 3) * a
    r2 = (pos * pos).sum(1)
    pos = pos[np.argsort(r2, kind="stable")[:n]]
    for _ in range(20):
        trial = pos + rng.normal(0.0, jitter, pos.shape)
        if n < 2 or not check:
            return trial
        d2 = ((trial[:, None, :] - trial[None, :, :]) ** 2).sum(-1) if n <= 3000 else None
        if d2 is None:
            return trial
        np.fill_diagonal(d2, np.inf)
        if d2.min() >= dmin * dmin:
            return trial
    return pos


def cluster_sizes(count, lo, hi, rng):
    """log-uniform sizes in [lo, hi], rounded."""
    return np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), count))).astype(int)


def batched_clusters(seed=3, count=1024, lo=13, hi=2000):
    """C3 part 1: `count` free Au clusters, log-uniform sizes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = cluster_sizes(count, lo, hi, rng)
    return [cluster(int(n), rng, check=False) for n in sizes]


def serve_stream(seed=4, rate=200.0, seconds=120.0, lo=13, hi=5000):
    """C4: Poisson arrivals of Au/Ag/Pt cluster jobs; 70 % FIRE relaxations,
    30 % 2000-step Langevin runs at U(300, 800) K.  Yields dicts with the
    arrival time (s), element, size, kind, temperature and seed."""
    rng = np.random.default_rng(seed)
    t = 0.0
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            return
        el = ("Au", "Ag", "Pt")[int(rng.integers(0, 3))]
        n = int(np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi)))))
        fire = rng.random() < 0.7
        yield dict(t=t, element=el, n=n, kind="fire" if fire else "md",
                   temp=float(rng.uniform(300.0, 800.0)), seed=1000 + k,
                   pos_seed=int(rng.integers(0, 2 ** 31)))
        k += 1
