"""Restatements of the reference's regression decks (examples/*/*.gms).

Each function builds the same system the deck builds -- atom order, box,
periodic flags, potentials, integrator and random stream -- so a run can be
compared with the golden rows of tests/golden/golden.json under the rule of
examples/test.sh.  The builders return plain numpy data plus a `setup`
callable that applies the deck's settings to any engine exposing the
oracle.System / gems_b200.System setter names, so the same deck drives the
oracle (CPU) and the CUDA path.
"""
import json
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")
_G = None


def golden():
    global _G
    if _G is None:
        with open(GOLDEN) as f:
            _G = json.load(f)
    return _G


def f32(x):
    """A default-real Fortran literal widened to real(dp) (e.g. e(47)%mass=107.87)."""
    return float(np.float32(x))


# Elements.F90 masses (single-precision literals assigned to real(dp))
MASS = {"H": f32(1.008), "He": f32(4.0032), "Ne": f32(20.183), "Si": f32(28.09),
        "Ag": f32(107.87), "Pt": f32(195.08), "Au": f32(196.97)}

# Fortran `dt=0.002` default (Program_Types.F90:53): a single-precision literal
DT_DEFAULT = f32(0.002)

# examples/test.sh pass rule: abs(sum((ref-new)^2) / sum(ref)) < 1e-6
def gems_rule(ref, new):
    ref = np.asarray(ref, dtype=np.float64)
    new = np.asarray(new, dtype=np.float64)
    return abs(np.sum((ref - new) ** 2) / np.sum(ref))


def e15(x):
    """Round like the E15.7 output format (7 significant digits)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    nz = x != 0
    mag = np.floor(np.log10(np.abs(x[nz]))) + 1
    out[nz] = np.round(x[nz] / 10.0 ** mag, 7) * 10.0 ** mag
    return out


# --------------------------------------------------------------- XYZ deck
def xyz_deck():
    """examples/XYZ/readxyz.gms: LJ energy of 6 frames, PBC box, no RNG."""
    g = golden()
    return dict(
        frames=[np.array(f, dtype=np.float64) for f in g["xyz_frames"]],
        box=(13.1399, 12.64396, 20.0000),
        lj=(0.1, 3.890898718140339, 10.0),
        ref=np.array(g["xyz_energy"])[:, 0],
    )


# --------------------------------------------------------------- LJ dimer
def lj_dimer_deck(kind="lj"):
    """examples/LJ/lj.gms (mass 3) and slj.gms (H atoms, the slj form with
    rs 1.108683): dimer scan (251 states) then 1000 VV steps."""
    g = golden()
    tau_ps = 0.01018
    d = dict(
        pos0=np.array([[1.0, 1.0, 1.0], [2.2, 1.0, 1.0]]),
        mass=3.0,
        box=(5.78, 5.78, 5.78),
        lj=(1.0, 0.890898718140339, 2.0),
        dt=0.002 * tau_ps,
        ref=np.array(g["lj_energy"]),
    )
    if kind == "slj":
        d.update(mass=MASS["H"], lj=None, slj=(1.0, 0.890898718140339, 1.108683), ref=np.array(g["slj_energy"]))
    return d


# --------------------------------------------------------------- SMA-TB bulk
def fcc_reply_positions(times=10):
    """bulk.gms atom order: 4-atom cell then `reply` along x, y, z (10 each).

    create_reply (Select_Create.F90:137-165) appends, for every atom of the
    current selection in order, its times-1 translated copies.
    """
    sel = [np.array(p, dtype=np.float64) for p in
           ([0, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0.5], [0.5, 0, 0.5])]
    for tras in ([1, 0, 0], [0, 1, 0], [0, 0, 1]):
        t = np.array(tras, dtype=np.float64)
        new = []
        for a in sel:
            for j in range(1, times):
                new.append(a + t * j)
        sel = sel + new
    return np.array(sel)


def bulk_deck():
    """examples/SMA-TB/bulk.gms: 4000 Ag fcc, boxed, no PBC, Ermak 1500 K."""
    g = golden()
    d0 = math.sqrt(0.5)
    fact = 2.89 / d0
    pos = fcc_reply_positions()
    pos = pos + np.array([1.0, 1.0, 1.0])
    pos = pos * fact            # expand about the origin
    box = tuple(12.0 * fact for _ in range(3))
    # baletto_2003.prm, Ag Ag line
    return dict(pos=pos, mass=MASS["Ag"], box=box, pbc=(False, False, False),
                smatb=AG_BALETTO, dt=DT_DEFAULT, temp=1500.0, gamma=1.0, nsteps=220,
                each=20, seed=123456, ref=np.array(g["smatb_bulk_energy"]))


AG_BALETTO = (0.1031, 1.1899, 10.85, 3.18, 2.89, 2.89 * math.sqrt(2.0), 2.89 * math.sqrt(3.0))


def md_deck():
    """examples/SMA-TB/md.gms: 13 Ag read from coords.xyz (no box: O(N^2)
    list), baletto_2003 Ag-Ag, `lbfgs` (lbfgs_minimizator, positions stay at
    the minimum), then Ermak 300 K, gamma 1/ps, dt 1 fs on the LCG stream of
    seed 123456, 1000 steps, a row every 100."""
    g = golden()
    return dict(pos=np.array(g["smatb_md_coords"], dtype=float), mass=MASS["Ag"], smatb=AG_BALETTO,
                dt=0.001, temp=300.0, gamma=1.0, nsteps=1000, each=100, seed=123456,
                ref=np.array(g["smatb_md_energy"]))


# --------------------------------------------------------------- NEB
NEB_BOX = (12.195, 15.0, 12.195)
# test.prm (examples/NEB): Au-Au Rossi 2005, Pt-Pt Cleri 1993, Au-Pt Logsdail 2009
NEB_PRM = {(0, 0): (0.2096, 1.8153, 10.139, 4.033, 2.8850, 2.8850 * math.sqrt(2.0), 2.8850 * math.sqrt(3.0)),
           (1, 1): (0.2975, 2.695, 10.612, 4.004, 3.924 / math.sqrt(2.0), 3.924, 3.924 * math.sqrt(3.0 / 2.0)),
           (0, 1): (0.25, 2.2, 10.42, 4.02, 2.830, 2.830 * math.sqrt(2.0), 2.830 * math.sqrt(3.0))}


def neb_deck():
    """examples/NEB/neb.gms: the 72-atom Au slab of configs/ref/gold_cube.xyz
    plus a Pt adatom at (0.2 Lx, 9.13, 0.2 Lz), all moved by 0.5 A, in a
    non-periodic 12.195 x 15 x 12.195 box; three fixed images, each relaxed
    by lbfgs after moving the Pt by (2, 0, 2) and then (2, 0, -2): images 1,
    15 and 30 of 30; neb_run 20 iterations, spring 5 eV/A^2."""
    g = golden()
    au = np.array(g["neb_gold_cube"], dtype=float)
    pt = np.array([[NEB_BOX[0] * 0.2, 9.13, NEB_BOX[2] * 0.2]])
    pos = np.vstack([au, pt]) + 0.5
    types = np.array([0] * len(au) + [1], dtype=np.int32)
    mass = np.array([MASS["Au"]] * len(au) + [MASS["Pt"]])
    return dict(pos=pos, types=types, mass=mass, box=NEB_BOX, prm=NEB_PRM, nimg=30, fixed=(0, 14, 29),
                moves=((2.0, 0.0, 2.0), (2.0, 0.0, -2.0)), k=5.0, iters=20, ref=np.array(g["neb_energy"]))


def neb_setup(s, d):
    s.set_box(d["box"], (False, False, False))
    for (a, b), prm in d["prm"].items():
        s.set_smatb(*prm, a, b)


def neb_fixed_images(s, d, relax):
    """The three fixed images: relax, store, move the Pt, relax, ...
    `relax(s)` runs the engine's L-BFGS on s."""
    imgs = np.zeros((d["nimg"],) + d["pos"].shape)
    relax(s)
    imgs[d["fixed"][0]] = s.pos
    for mv, k in zip(d["moves"], d["fixed"][1:]):
        p = s.pos
        p[-1] += mv
        s.set_pos(p)
        relax(s)
        imgs[k] = s.pos
    return imgs


def neb_rows(images, energy_ev):
    """write_neb (src/NEB.f90:376-414): per image the path length fraction
    and its potential energy (eV); energy_ev is a function of an image's
    positions or the energies themselves."""
    gc = [0.0]
    for i in range(1, len(images)):
        gc.append(gc[-1] + float(np.sqrt(((images[i] - images[i - 1]) ** 2).sum())))
    gc = np.array(gc) / gc[-1]
    e = [energy_ev(im) for im in images] if callable(energy_ev) else list(energy_ev)
    return np.c_[gc, np.asarray(e, dtype=float)]


def neb_rule(ref, got):
    """examples/test.sh for NEB: sum of squared differences of the first two
    columns over the sum of the first column, < 1e-4."""
    a = ((ref[:, 1] - got[:, 1]) ** 2).sum() + ((ref[:, 0] - got[:, 0]) ** 2).sum()
    return abs(a / ref[:, 0].sum())


# --------------------------------------------------------------- NPT
def npt_lgf_deck():
    """examples/NPT/lgf.gms: fcc 6^3 (864 atoms of mass 1.008) expanded by
    sqrt(2) in a 6 sqrt(2) periodic box, moved by 0.2; slj(1 eV, 2^(-1/6) A,
    rs 1.108683); G-JF constant pressure and temperature (piston_lgf xyz*) at
    0.3 e0/kB, particle friction 1/tau, piston friction 1e-4/tau, piston mass
    1e-5, pressure 0.1 e0/r0^3 given in atm; dt = 0.01 tau (tau = 0.01018 ps);
    100 steps on the LCG stream of seed 123456, a row every 10.  The deck
    sets `box mic F` (ghost atoms); at this box size the minimum image gives
    the same interactions and virial."""
    g = golden()
    f = math.sqrt(2.0)
    pos = fcc_reply_positions(6) * f + 0.2
    tau = 0.01018
    return dict(pos=pos, mass=MASS["H"], box=(6.0 * f,) * 3, slj=(1.0, 2.0 ** (-1.0 / 6.0), 1.108683),
                dt=0.01 * tau, temp=0.3 * 11604.45, press_atm=0.1 * 1581225.25240563, pgama0=1.0 / tau,
                pgamav=0.0001 / tau, pmass=0.00001, nsteps=100, each=10, seed=123456,
                ref_energy=np.array(g["npt_lgf_energy"]), ref_press=np.array(g["npt_lgf_press"]),
                ref_virial=np.array(g["npt_lgf_virial"]))


def npt_axes_deck(kind):
    """examples/NPT/lgf_flex.gms ("flex": a G-JF piston on each of x, y, z,
    piston friction 1/tau and mass 0.1) and lgf_x.gms ("x": a piston on x
    at 1 e0/r0^3, Ermak on y and z at 1/tau): the lgf.gms crystal and
    potential otherwise.  `axes` lists the per-coordinate integrators in
    deck order: ("lgf", axis, T, gamma0, P atm, gammav, pmass) or
    ("ermak", axis, T, gamma)."""
    g = golden()
    d = npt_lgf_deck()
    tau = 0.01018
    T = 0.3 * 11604.45
    e0r0 = 1581225.25240563
    if kind == "flex":
        d["axes"] = [("lgf", k, T, 1.0 / tau, 0.1 * e0r0, 1.0 / tau, 0.1) for k in range(3)]
        d.update(ref_energy=np.array(g["npt_flex_energy"]), ref_press=np.array(g["npt_flex_press"]),
                 ref_virial=np.array(g["npt_flex_virial"]), ref_box=None)
    else:
        d["axes"] = [("lgf", 0, T, 1.0 / tau, 1.0 * e0r0, 1.0 / tau, 0.1),
                     ("ermak", 1, T, 1.0 / tau), ("ermak", 2, T, 1.0 / tau)]
        d.update(ref_energy=np.array(g["npt_x_energy"]), ref_press=np.array(g["npt_x_press"]),
                 ref_virial=None, ref_box=np.array(g["npt_x_box"]))
    return d


def npt_axes_setup(s, d, rng):
    """The per-coordinate integrators of an npt_axes_deck, oracle or GPU
    (`rng` is the oracle's stream or a GPU seed)."""
    s.set_box(d["box"], (True, True, True))
    s.set_slj(*d["slj"])
    for a in d["axes"]:
        if a[0] == "lgf":
            s.add_lgf_axis(a[1], d["dt"], a[2], a[4], a[3], a[5], a[6], rng)
        else:
            s.add_ermak_axis(a[1], d["dt"], a[3], a[2], rng)


def npt_lkd_deck():
    """The lgf.gms crystal, potential and targets under `evolve piston_lkd`
    (piston friction 1e-4/tau, piston mass 1e-5).  The reference ships no
    golden file for this integrator."""
    d = npt_lgf_deck()
    d["lkd"] = True
    return d


def npt_axes_pairs(d, n):
    """LCG pairs one step draws: a piston takes 1 + n, an Ermak coordinate n."""
    return sum(1 + n if a[0] == "lgf" else n for a in d["axes"])


def npt_setup(s, d, rng):
    s.set_box(d["box"], (True, True, True))
    s.set_slj(*d["slj"])
    if d.get("lkd"):
        s.set_lkd(d["dt"], d["temp"], d["press_atm"], d["pgama0"], d["pgamav"], d["pmass"], rng)
    else:
        s.set_lgf(d["dt"], d["temp"], d["press_atm"], d["pgama0"], d["pgamav"], d["pmass"], rng)


def npt_run(s, d, rng, nsteps=None, each=None, feed=None, boxes=None):
    """dinamic with per-step rows of (Epot, Ekin, Etot in eV, T), pressure
    (atm) and virial (eV).  `feed(s, normals)` hands each step's LCG normals
    to an engine in parity mode (the pairs of one step in the order the
    reference draws them); `boxes`, a list, receives the box lengths of each
    row."""
    nsteps = nsteps or d["nsteps"]
    each = each or d["each"]
    s.interact()
    E, P, V = [], [], []
    for ns in range(1, nsteps + 1):
        if feed is not None:
            if "axes" in d:
                pairs = npt_axes_pairs(d, s.n)
            else:
                pairs = 6 * s.n + 2 if d.get("lkd") else 1 + 3 * s.n
            feed(s, rng.rang_stream(pairs))
        s.stepa()
        s.interact()
        s.stepb()
        if ns % each == 0:
            ek, t = s.kin()
            ep = s.epot_sum()
            E.append([ep, ek, ep + ek, t])
            P.append(s.pressure_atm())
            V.append(s.virial_ev())
            if boxes is not None:
                boxes.append(s.box_now())
    return np.array(E), np.array(P), np.array(V)


# --------------------------------------------------------------- NVE / NVT
def he_ne_gas(rng):
    """v_verlet.gms / ermak.gms set-up: `fill 100 2.6` He then Ne in 50^3."""
    box = (50.0, 50.0, 50.0)
    he = rng.fill(np.zeros((0, 3)), [], 100, 2.6, box)
    ne = rng.fill(he, [2.6] * 100, 100, 2.6, box)
    pos = np.concatenate([he, ne])
    types = np.array([0] * 100 + [1] * 100, dtype=np.int32)
    mass = np.array([MASS["He"]] * 100 + [MASS["Ne"]] * 100)
    return pos, types, mass, box


def plj_params():
    """The three plj groups of v_verlet.gms (He-He, Ne-Ne, He-Ne)."""
    cal_ev = 2.61144768e19
    na = 6.0221417930e23
    kcalmol_ev = cal_ev / na * 1000.0
    return {
        (0, 0): (0.021270 * kcalmol_ev, 1.4800),
        (1, 1): (0.086000 * kcalmol_ev, 1.5300),
        (0, 1): (math.sqrt(0.086000 * 0.021270) * kcalmol_ev, 0.5 * (1.5300 + 1.4800)),
    }


def lj_dimer_rows(sys_factory, ui_ev, kind="lj"):
    """Run the lj.gms or slj.gms deck on an engine; returns (rows, golden rows)."""
    d = lj_dimer_deck(kind)
    pos = d["pos0"].copy()
    s = sys_factory(pos, d["mass"])
    s.set_box(d["box"], (False, False, False))
    if d["lj"] is not None:
        s.set_lj(*d["lj"])
    else:
        s.set_slj(*d["slj"])
    rows = []

    def state():
        s.set_pos(pos)
        s.interact()
        ek, _ = s.kin()
        ep = s.epot_sum()
        rows.append([ep * ui_ev, ek * ui_ev, (ep + ek) * ui_ev])

    state()
    for mv in (-1.2, 0.9):
        pos[1, 0] = pos[1, 0] + mv
    for _ in range(250):
        pos[1, 0] = pos[1, 0] + 0.01
        state()
    for mv in (-2.5, -0.9, 1.2):
        pos[1, 0] = pos[1, 0] + mv
    s.set_pos(pos)
    s.set_vv(d["dt"])
    r = s.dinamica(1000, 10)
    return np.concatenate([np.array(rows), r[:, :3]]), d["ref"]


# wca, sm1 and feels decks of examples/LJ (FP64 H atoms, mass 1.008)
WCA_SIGMA = 0.890898718140339
SLJ_PRM = (1.0, 0.890898718140339, 1.108683)


def lj_family_rows(sys_factory, ui_ev, kind):
    """Run examples/LJ/wca.gms, sm1.gms or feels.gms on an engine.

    sys_factory(pos, mass, types, ntypes) makes the system; one atom type per
    group of the deck, so that a one-sided `feels` pair is a pair of types.
    Returns (rows of epot, ekin, etot in eV, golden rows)."""
    g = golden()
    rows = []
    mass = MASS["H"]

    def state(s, pos):
        s.set_pos(pos)
        s.interact()
        ek, _ = s.kin()
        ep = s.epot_sum()
        rows.append([ep * ui_ev, ek * ui_ev, (ep + ek) * ui_ev])

    if kind == "wca":
        # group 2 = atom 2 feels group 3 = atom 1: `interact 2 feels 3 wca`
        pos = np.array([[1.0, 1.0, 1.0], [2.2, 1.0, 1.0]])
        s = sys_factory(pos.copy(), mass, np.array([0, 1]), 2)
        s.set_box((5.78, 5.78, 5.78), (False, False, False))
        s.set_wca(1.0, WCA_SIGMA, ti=1, tj=0)
        s.set_feels(1, 0)
        state(s, pos)
        pos[1, 0] += -1.2
        pos[1, 0] += WCA_SIGMA
        state(s, pos)
        pos[1, 0] += -WCA_SIGMA
        pos[1, 0] += 0.9
        for _ in range(250):
            pos[1, 0] += 0.01
            state(s, pos)
        for mv in (-2.5, -0.9, 0.95):
            pos[1, 0] += mv
        s.set_pos(pos)
        s.set_vv(0.002 * 0.01018)
        r = s.dinamica(1000, 10)
        ref = g["wca_energy"]
    elif kind == "sm1":
        # no box: the O(N^2) list; both atoms start on the same site
        pos = np.array([[1.0, 1.0, 1.0], [1.0, 1.0, 1.0]])
        s = sys_factory(pos.copy(), mass, np.array([0, 0]), 1)
        s.set_sm1(1.0, 2.0, 0.01)
        state(s, pos)
        for _ in range(300):
            pos[1, 0] += 0.01
            state(s, pos)
        pos[1, 0] += -2.0
        s.set_pos(pos)
        # set_cm_vel (Set_Properties.f90:981-997) of group 2 = atom 2
        s.set_vel(np.array([[0.0, 0.0, 0.0], [10.0, 0.0, 0.0]]))
        s.set_vv(0.001)
        r = s.dinamica(1000, 1)
        ref = g["sm1_energy"]
    elif kind == "feels":
        # types: 0 = atoms 1, 3; 1 = atoms 2, 4 (group 3); 2 = atom 5 (group 4)
        pos = np.array([[1.0, 1.0, 1.0], [2.2, 1.0, 1.0], [1.0, 1.0, 5.0],
                        [2.2, 1.0, 5.0], [3.4, 1.0, 1.0]])
        s = sys_factory(pos.copy(), mass, np.array([0, 1, 0, 1, 2]), 3)
        s.set_box((5.78, 5.78, 5.78), (False, False, False))
        for a, b in ((0, 0), (0, 1), (1, 1)):   # interact 2 with 2 slj
            s.set_slj(*SLJ_PRM, ti=a, tj=b)
        s.set_slj(*SLJ_PRM, ti=2, tj=1)          # interact 4 feels 3 slj
        s.set_feels(2, 1)
        state(s, pos)
        s.set_vv(0.002 * 0.01018)
        r = s.dinamica(1000, 10)
        ref = g["feels_energy"]
    else:
        raise ValueError(kind)
    return np.concatenate([np.array(rows), r[:, :3]]), np.array(ref)


def chp_records(data):
    """Fortran unformatted sequential records (4-byte length before and after)."""
    import struct
    out, at = [], 0
    while at < len(data):
        (m,) = struct.unpack_from("<i", data, at)
        (m2,) = struct.unpack_from("<i", data, at + 4 + m)
        assert m == m2
        out.append(data[at + 4:at + 4 + m])
        at += 8 + m
    return out


def chp_atoms(data, n):
    """The per-atom records of a GEMS .chp file as a (6, n, 3) array: pos,
    vel, acel, acel2, acel3, acel4 (write_chp, Checkpoint.F90:175-184)."""
    import struct
    r = chp_records(data)[-6 * n:]
    return np.array([[struct.unpack("<3d", r[6 * i + k]) for i in range(n)] for k in range(6)])


def he_ne_setup(O):
    """NVE/NVT initial state from the oracle's stream (fill, box move,
    tempgdist 300); returns positions, velocities, types, masses, box, rng."""
    rng = O.Rng(123456)
    pos, types, mass, box = he_ne_gas(rng)
    s = O.System(pos, mass, types, 2)
    s.set_box(box, (True, True, True))
    for (a, b), (e, sg) in plj_params().items():
        s.set_lj(e, sg, 10.0, a, b, shifted_force=True)
    s.remove_cm()
    s.gdist(rng, 300.0)
    return pos, s.vel, types, mass, box, rng


def apply_plj(s):
    for (a, b), (e, sg) in plj_params().items():
        s.set_lj(e, sg, 10.0, a, b, shifted_force=True)


def ermak_parity_run(s, rng, nsteps, each):
    """dinamic with the Ermak normals taken from the LCG stream (rang pairs in
    atom order), fed to the engine step by step."""
    s.interact()
    rows = []
    for ns in range(1, nsteps + 1):
        s.set_ermak_normals(rng.rang_stream(3 * s.n))
        s.stepa()
        s.interact()
        s.stepb()
        if ns % each == 0:
            ek, t = s.kin()
            ep = s.epot_sum()
            rows.append([ep, ek, ep + ek, t])
    return np.array(rows)


def repex_rows(O):
    """examples/RepExchange/lj.gms on the oracle: 4 replicas (one per MPI rank
    of the reference, each with its own LCG stream seeded 123456*rank), Ermak
    at 30/35/40/45, `dinamica 1000`, `out state`, then `partemp2 100 100`
    with the swap rule of parallel_tempering2 (src/ReplicaExchange.f90:55-138).
    Like the reference, a swap exchanges positions and velocities (not acel)
    and rescales the velocities by sqrt(T_self/T_partner)."""
    import math
    tau_ps = 0.01018
    dt = 0.002 * tau_ps
    gam = 1.0 / tau_ps
    kB_ui = O.lib().orc_kB_ui()
    reps = []
    for pc in range(4):
        rng = O.Rng(123456 * pc)
        s = O.System(np.array([[1.0, 1, 1], [2.2, 1, 1]]) + 1.0, 3.0)
        s.set_box((5.78,) * 3, (False,) * 3)
        s.set_lj(1.0, 0.890898718140339, 2.0)
        T = pc * 5.0 + 30
        s.gdist(rng, T)
        s.set_ermak(dt, gam, T, rng)
        reps.append((s, rng, T))
    for s, _, _ in reps:
        s.dinamica(1000, 0)
    rows = [[] for _ in range(4)]
    for pc, (s, _, _) in enumerate(reps):
        e = s.interact()
        ek, _ = s.kin()
        rows[pc].append(e * O.UI_EV)
    for ns in range(1, 101):
        for pc, (s, _, _) in enumerate(reps):
            rows[pc] += list(s.dinamica(100, 10)[:, 0])
        par = 1 if ns % 2 == 0 else -1
        ep = [s.interact() for s, _, _ in reps]
        for pc in range(4):
            p = pc + par if pc % 2 == 0 else pc - par
            if p < 0 or p >= 4 or p < pc:
                continue
            (a, ra, ta), (b, _, tb) = reps[pc], reps[p]
            du = (ep[p] - ep[pc]) * (1.0 / (kB_ui * ta) - 1.0 / (kB_ui * tb))
            if du > 0 and not ra.ranu() < math.exp(-du):
                continue
            pa, va, pb, vb = a.pos, a.vel, b.pos, b.vel
            a.set_pos(pb)
            a.set_vel(vb * math.sqrt(ta / tb))
            b.set_pos(pa)
            b.set_vel(va * math.sqrt(tb / ta))
    return [np.array(r) for r in rows]
