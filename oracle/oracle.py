"""ctypes wrapper of the FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: a CPU restatement of the GEMS force/neighbour hot
path that the tests compare the CUDA path against, and the timed CPU baseline.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module;
the product library never does.

Positions, velocities and forces use the GEMS interleaved layout
[x1, y1, z1, x2, ...] in internal units (Angstrom, uma, ps); energies are
returned in internal units unless a function says eV.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_long
_p = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so from oracle/gems_oracle.cpp (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(_HERE, "gems_oracle.cpp")
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        build()
    L = ctypes.CDLL(_LIB)
    sig = {
        "orc_ev_ui": (_d, []), "orc_kB_ui": (_d, []),
        "orc_max_threads": (_i, []), "orc_set_threads": (None, [_i]),
        "orc_rng_new": (_p, [_i]), "orc_rng_free": (None, [_p]),
        "orc_ranu": (_d, [_p]), "orc_rang": (None, [_p, _dp, _dp]),
        "orc_rang_stream": (None, [_p, _l, _dp]),
        "orc_rng_state": (None, [_p, _ip]),
        "orc_fill": (_i, [_p, _i, _dp, _dp, _i, _d, _dp, _dp]),
        "orc_sys_new": (_p, [_i]), "orc_sys_free": (None, [_p]),
        "orc_set_pos": (None, [_p, _dp]), "orc_get_pos": (None, [_p, _dp]),
        "orc_set_vel": (None, [_p, _dp]), "orc_get_vel": (None, [_p, _dp]),
        "orc_set_acel": (None, [_p, _dp]), "orc_get_acel": (None, [_p, _dp]),
        "orc_get_force": (None, [_p, _dp]),
        "orc_get_epot_atoms": (None, [_p, _dp]),
        "orc_get_band": (None, [_p, _dp]),
        "orc_set_mass": (None, [_p, _dp]),
        "orc_set_types": (None, [_p, _ip, _i]),
        "orc_set_box": (None, [_p, _i, _dp, _ip]),
        "orc_set_mic": (None, [_p, _i]),
        "orc_set_skin": (None, [_p, _d]),
        "orc_set_skin_mode": (None, [_p, _i]),
        "orc_set_half": (None, [_p, _i]),
        "orc_set_capacity": (None, [_p, _i]),
        "orc_set_lj": (None, [_p, _i, _i, _d, _d, _d, _i, _d]),
        "orc_set_smatb": (None, [_p, _i, _i, _d, _d, _d, _d, _d, _d, _d]),
        "orc_set_tersoff": (None, [_p, _dp]),
        "orc_smatb_coeffs": (None, [_p, _i, _i, _dp]),
        "orc_interact": (_d, [_p, _ip]),
        "orc_update": (None, [_p]),
        "orc_nupd": (_l, [_p]),
        "orc_status": (_i, [_p]),
        "orc_list_cap": (_i, [_p]),
        "orc_uses_cells": (_i, [_p, _ip]),
        "orc_get_list": (None, [_p, _ip, _ip]),
        "orc_set_vv": (None, [_p, _d]),
        "orc_set_ermak": (None, [_p, _d, _d, _d, _p]),
        "orc_ermak_consts": (None, [_p, _dp]),
        "orc_set_ext_normals": (None, [_p, _dp]),
        "orc_set_fire": (None, [_p, _d, _d]),
        "orc_fire_dt": (_d, [_p]),
        "orc_fmax": (_d, [_p]),
        "orc_stepa": (None, [_p]), "orc_stepb": (None, [_p]),
        "orc_do_pbc": (None, [_p]),
        "orc_kin": (None, [_p, _dp, _dp]),
        "orc_epot_sum": (_d, [_p]),
        "orc_gdist": (None, [_p, _p, _d]),
        "orc_remove_cm": (None, [_p]),
        "orc_dinamica": (_i, [_p, _i, _i, _dp]),
        "orc_fire_relax": (_i, [_p, _d, _i, _dp]),
        "orc_lbfgs": (_i, [_p, _i, _d, _d, _i, _ip, _ip, _dp]),
        "orc_neb": (_d, [_p, _i, _dp, _ip, _i, _d, _i]),
        "orc_set_slj": (None, [_p, _i, _i, _d, _d, _d]),
        "orc_set_wca": (None, [_p, _i, _i, _d, _d]),
        "orc_set_sm1": (None, [_p, _i, _i, _d, _d, _d]),
        "orc_set_feels": (None, [_p, _i, _i]),
        "orc_set_pred_corr": (None, [_p, _d]),
        "orc_set_brownian": (None, [_p, _d, _d, _d, _p]),
        "orc_set_scalvel": (None, [_p, _d, _i, _d]),
        "orc_set_andersen": (None, [_p, _d, _d, _p]),
        "orc_clear_thermostat": (None, [_p]),
        "orc_get_derivs": (None, [_p, _dp]),
        "orc_set_derivs": (None, [_p, _dp]),
        "orc_set_lgf": (None, [_p, _d, _d, _d, _d, _d, _d, _p]),
        "orc_virial_ev": (None, [_p, _dp]),
        "orc_add_lgf_axis": (None, [_p, _i, _d, _d, _d, _d, _d, _d, _p]),
        "orc_add_ermak_axis": (None, [_p, _i, _d, _d, _d, _p]),
        "orc_set_lkd": (None, [_p, _d, _d, _d, _d, _d, _d, _p]),
        "orc_rng_set_state": (None, [_p, _i, _i, _i]),
        "orc_piston_state": (None, [_p, _dp, _dp]),
        "orc_pressure_atm": (None, [_p, _dp]),
        "orc_get_box": (None, [_p, _dp]),
        "orc_atm_ui": (_d, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a, ct=_d):
    return a.ctypes.data_as(ctypes.POINTER(ct))


EV_UI = None
UI_EV = None
KB_UI = None


def _units():
    global EV_UI, UI_EV, KB_UI
    if EV_UI is None:
        EV_UI = lib().orc_ev_ui()
        UI_EV = 1.0 / EV_UI
        KB_UI = lib().orc_kB_ui()


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


class Rng:
    """LCG + polar Box-Muller stream of Random.F90:145-250."""

    def __init__(self, seed):
        self.h = lib().orc_rng_new(int(seed))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_rng_free(self.h)
            self.h = None

    def ranu(self):
        return lib().orc_ranu(self.h)

    def rang(self):
        a, b = _d(), _d()
        lib().orc_rang(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def rang_stream(self, npairs):
        out = np.empty(2 * int(npairs), dtype=np.float64)
        lib().orc_rang_stream(self.h, int(npairs), _ptr(out))
        return out

    def set_state(self, idum, iy, ix):
        """lcg_read_chpseed: resume from a checkpoint's (idum, iy, ix)."""
        lib().orc_rng_set_state(self.h, int(idum), int(iy), int(ix))

    def chp_state(self):
        """(idum, iy, ix) in the order write_chpseed stores them."""
        st = self.state()
        return int(st[0]), int(st[2]), int(st[1])

    def state(self):
        st = np.zeros(4, dtype=np.int32)
        lib().orc_rng_state(self.h, _ptr(st, _i))
        return st

    def fill(self, pos_old, sig_old, num, sigma, frame, origin=(0.0, 0.0, 0.0)):
        """create_fill: returns the num new positions (num x 3)."""
        n_old = len(sig_old)
        buf = np.zeros(3 * (n_old + num), dtype=np.float64)
        if n_old:
            buf[: 3 * n_old] = np.asarray(pos_old, dtype=np.float64).ravel()
        so = np.ascontiguousarray(sig_old, dtype=np.float64)
        fr = np.asarray(frame, dtype=np.float64)
        og = np.asarray(origin, dtype=np.float64)
        r = lib().orc_fill(self.h, n_old, _ptr(buf), _ptr(so) if n_old else None,
                           int(num), float(sigma), _ptr(fr), _ptr(og))
        if r < 0:
            raise RuntimeError("fill: max iteration reached, no space was found")
        return buf[3 * n_old:].reshape(num, 3)


class System:
    """One simulated system of the oracle (mirrors a GEMS group + intergroup)."""

    def __init__(self, pos, mass, types=None, ntypes=1):
        _units()
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        self.n = pos.shape[0]
        self.h = lib().orc_sys_new(self.n)
        self.set_pos(pos)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, dtype=np.float64), (self.n,)))
        lib().orc_set_mass(self.h, _ptr(m))
        t = np.zeros(self.n, dtype=np.int32) if types is None else np.ascontiguousarray(types, dtype=np.int32)
        self._types = t
        lib().orc_set_types(self.h, _ptr(t, _i), int(ntypes))
        self._keep = []

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_sys_free(self.h)
            self.h = None

    # state -------------------------------------------------------------
    def _get(self, fn, k=3):
        out = np.empty(self.n * k, dtype=np.float64)
        fn(self.h, _ptr(out))
        return out.reshape(self.n, k) if k == 3 else out

    def set_pos(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        lib().orc_set_pos(self.h, _ptr(x))

    def set_vel(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        lib().orc_set_vel(self.h, _ptr(v))

    def set_acel(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        lib().orc_set_acel(self.h, _ptr(a))

    @property
    def pos(self):
        return self._get(lib().orc_get_pos)

    @property
    def vel(self):
        return self._get(lib().orc_get_vel)

    @property
    def acel(self):
        return self._get(lib().orc_get_acel)

    @property
    def force(self):
        return self._get(lib().orc_get_force)

    @property
    def epot_atoms(self):
        return self._get(lib().orc_get_epot_atoms, 1)

    @property
    def band(self):
        return self._get(lib().orc_get_band, 1)

    # setup ---------------------------------------------------------------
    def set_box(self, L=None, pbc=(True, True, True)):
        if L is None:
            lib().orc_set_box(self.h, 0, None, None)
            return
        Lb = np.asarray(L, dtype=np.float64)
        pb = np.asarray([1 if b else 0 for b in pbc], dtype=np.int32)
        lib().orc_set_box(self.h, 1, _ptr(Lb), _ptr(pb, _i))

    def set_mic(self, mic):
        lib().orc_set_mic(self.h, 1 if mic else 0)

    def set_skin(self, skin):
        lib().orc_set_skin(self.h, float(skin))

    def set_skin_mode(self, mic):
        """True: skin test on minimum-image displacements (fewer rebuilds,
        same forces); False: the reference's raw displacements (default)."""
        lib().orc_set_skin_mode(self.h, 1 if mic else 0)

    def set_half(self, half):
        lib().orc_set_half(self.h, 1 if half else 0)

    def set_capacity(self, cap):
        lib().orc_set_capacity(self.h, int(cap))

    def set_lj(self, e, s, rc, ti=0, tj=0, shifted_force=False, eshift=0.0):
        lib().orc_set_lj(self.h, ti, tj, e, s, rc, 1 if shifted_force else 0, eshift)

    def set_pred_corr(self, dt):
        """`evolve pred_corr_5`: the fifth-order Nordsieck predictor-corrector."""
        lib().orc_set_pred_corr(self.h, float(dt))

    def set_brownian(self, dt, temp, gama, rng):
        """`evolve brownian temp gama` (set_cbrownian / cbrownian)."""
        self._rng = rng
        lib().orc_set_brownian(self.h, float(dt), float(temp), float(gama), rng.h)

    def set_scalvel(self, temp, steps, upto=None):
        """`evolve scalvel temp steps` (or scalvel_after with upto), run
        after the integrator's step b."""
        lib().orc_set_scalvel(self.h, float(temp), int(steps), -1.0 if upto is None else float(upto))

    def set_andersen(self, temp, nu, rng):
        """`evolve andersen temp nu`, run after the integrator's step b."""
        self._rng2 = rng
        lib().orc_set_andersen(self.h, float(temp), float(nu), rng.h)

    def clear_thermostat(self):
        lib().orc_clear_thermostat(self.h)

    def derivs(self):
        """acel, acel2, acel3, acel4 as a (4, n, 3) array."""
        out = np.empty((4, self.n, 3), dtype=np.float64)
        lib().orc_get_derivs(self.h, _ptr(out))
        return out

    def set_derivs(self, d):
        a = np.ascontiguousarray(d, dtype=np.float64).reshape(4, self.n, 3)
        lib().orc_set_derivs(self.h, _ptr(a))

    def set_wca(self, e, s, ti=0, tj=0):
        """wca_set: LJ cut at its minimum and shifted up by e."""
        lib().orc_set_wca(self.h, int(ti), int(tj), float(e), float(s))

    def set_sm1(self, r1, r2, e, ti=0, tj=0):
        """sm1_set: smooth step of depth e (eV) from r1 to r2."""
        lib().orc_set_sm1(self.h, int(ti), int(tj), float(r1), float(r2), float(e))

    def set_feels(self, ti, tj):
        """`interact g1 feels g2`: the pair (ti, tj) acts on type ti only."""
        lib().orc_set_feels(self.h, int(ti), int(tj))

    def set_smatb(self, A, xi, p, q, r0, rci, rce, ti=0, tj=0):
        lib().orc_set_smatb(self.h, ti, tj, A, xi, p, q, r0, rci, rce)

    def set_tersoff(self, prm):
        a = np.ascontiguousarray(prm, dtype=np.float64)
        self._keep.append(a)
        lib().orc_set_tersoff(self.h, _ptr(a))

    def smatb_coeffs(self, ti=0, tj=0):
        out = np.empty(6, dtype=np.float64)
        lib().orc_smatb_coeffs(self.h, ti, tj, _ptr(out))
        return out

    # compute -------------------------------------------------------------
    def interact(self):
        """Forces + energy (internal units); first call builds the list."""
        rb = _i()
        e = lib().orc_interact(self.h, ctypes.byref(rb))
        return e

    def update(self):
        lib().orc_update(self.h)

    @property
    def nupd(self):
        return lib().orc_nupd(self.h)

    @property
    def status(self):
        return lib().orc_status(self.h)

    def uses_cells(self):
        nc = np.zeros(3, dtype=np.int32)
        u = lib().orc_uses_cells(self.h, _ptr(nc, _i))
        return bool(u), tuple(int(v) for v in nc)

    def neighbour_list(self):
        """(nn, list) with list shaped (cap, n) column-major like list(i,m)."""
        cap = lib().orc_list_cap(self.h)
        nn = np.empty(self.n, dtype=np.int32)
        lst = np.empty(cap * self.n, dtype=np.int32)
        lib().orc_get_list(self.h, _ptr(nn, _i), _ptr(lst, _i))
        return nn, lst.reshape(cap, self.n)

    def pair_set(self):
        """Sorted (i, j) pairs of the current list as an int64 key array."""
        nn, lst = self.neighbour_list()
        i_idx = np.concatenate([np.full(c, i, dtype=np.int64) for i, c in enumerate(nn)]) if self.n else np.zeros(0, np.int64)
        j_idx = np.concatenate([lst[: c, i].astype(np.int64) for i, c in enumerate(nn)]) if self.n else np.zeros(0, np.int64)
        return np.sort(i_idx * self.n + j_idx)

    # integrators -----------------------------------------------------------
    def set_vv(self, dt):
        lib().orc_set_vv(self.h, float(dt))

    def set_ermak(self, dt, gama, temp, rng):
        self._rng = rng
        lib().orc_set_ermak(self.h, float(dt), float(gama), float(temp), rng.h if rng else None)

    def ermak_consts(self):
        out = np.empty(8, dtype=np.float64)
        lib().orc_ermak_consts(self.h, _ptr(out))
        return out

    def set_ext_normals(self, nrm):
        """Use an external normal stream (6 per atom) in ermak_a."""
        if nrm is None:
            lib().orc_set_ext_normals(self.h, None)
            return
        a = np.ascontiguousarray(nrm, dtype=np.float64)
        self._ext = a
        lib().orc_set_ext_normals(self.h, _ptr(a))

    def set_fire(self, dt0, dtmax):
        lib().orc_set_fire(self.h, float(dt0), float(dtmax))

    def stepa(self):
        lib().orc_stepa(self.h)

    def stepb(self):
        lib().orc_stepb(self.h)

    def do_pbc(self):
        lib().orc_do_pbc(self.h)

    def kin(self):
        ek, t = _d(), _d()
        lib().orc_kin(self.h, ctypes.byref(ek), ctypes.byref(t))
        return ek.value, t.value

    def epot_sum(self):
        return lib().orc_epot_sum(self.h)

    def gdist(self, rng, temp):
        lib().orc_gdist(self.h, rng.h, float(temp))

    def remove_cm(self):
        lib().orc_remove_cm(self.h)

    def dinamica(self, nsteps, each):
        nrows = nsteps // each if each > 0 else 0
        rows = np.zeros(4 * max(nrows, 1), dtype=np.float64)
        nr = lib().orc_dinamica(self.h, int(nsteps), int(each), _ptr(rows))
        return rows[: 4 * nr].reshape(nr, 4)

    def fire_relax(self, fmax_tol, maxit):
        fm = _d()
        it = lib().orc_fire_relax(self.h, float(fmax_tol), int(maxit), ctypes.byref(fm))
        return it, fm.value

    def fmax(self):
        return lib().orc_fmax(self.h)

    def set_slj(self, e, sg, rs, ti=0, tj=0):
        lib().orc_set_slj(self.h, int(ti), int(tj), float(e), float(sg), float(rs))

    def set_lgf(self, dt, temp, press_atm, pgama0, pgamav, pmass, rng=None):
        """set_lgf (G-JF constant pressure): press in atm as the deck gives it."""
        self._rng = rng
        lib().orc_set_lgf(self.h, float(dt), float(temp), float(press_atm), float(pgama0), float(pgamav),
                          float(pmass), rng.h if rng is not None else None)

    def set_lkd(self, dt, temp, press_atm, pgama0, pgamav, pmass, rng):
        """`evolve piston_lkd`: the Langevin piston of Kolb & Dunweg."""
        self._rng = rng
        lib().orc_set_lkd(self.h, float(dt), float(temp), float(press_atm), float(pgama0), float(pgamav),
                          float(pmass), rng.h)

    def add_lgf_axis(self, axis, dt, temp, press_atm, pgama0, pgamav, pmass, rng):
        """`evolve piston_lgf x|y|z`: a G-JF piston on one box length."""
        self._rng = rng
        lib().orc_add_lgf_axis(self.h, int(axis), float(dt), float(temp), float(press_atm), float(pgama0),
                               float(pgamav), float(pmass), rng.h)

    def add_ermak_axis(self, axis, dt, gama, temp, rng):
        """`evolve ermak_x|y|z`: Ermak dynamics of one coordinate."""
        self._rng = rng
        lib().orc_add_ermak_axis(self.h, int(axis), float(dt), float(gama), float(temp), rng.h)

    def piston_state(self):
        """(pistonf[3], pvel[3]) after the last step, internal units."""
        pf, pv = np.zeros(3), np.zeros(3)
        lib().orc_piston_state(self.h, _ptr(pf), _ptr(pv))
        return pf, pv

    def virial_ev(self):
        out = np.zeros(9)
        lib().orc_virial_ev(self.h, _ptr(out))
        return out

    def pressure_atm(self):
        out = np.zeros(9)
        lib().orc_pressure_atm(self.h, _ptr(out))
        return out

    def box_now(self):
        out = np.zeros(3)
        lib().orc_get_box(self.h, _ptr(out))
        return out

    def neb(self, images, fixed, k_ev, iters):
        """neb_run: images (nimg x n x 3; the fixed ones set) -> (relaxed
        images, dt).  `fixed` holds 0-based image indices."""
        im = np.ascontiguousarray(images, dtype=np.float64).copy()
        fx = np.ascontiguousarray(fixed, dtype=np.int32)
        dt = lib().orc_neb(self.h, im.shape[0], _ptr(im), _ptr(fx, ctypes.c_int), len(fx), float(k_ev), int(iters))
        return im, dt

    def lbfgs(self, m=5, eps=1e-8, xtol=1e-15, itermax=1000):
        """lbfgs_minimizator: minimise in place; returns (iflag, iterations,
        function evaluations, f in eV)."""
        it, nf, fm = ctypes.c_int(), ctypes.c_int(), _d()
        flag = lib().orc_lbfgs(self.h, int(m), float(eps), float(xtol), int(itermax), ctypes.byref(it),
                               ctypes.byref(nf), ctypes.byref(fm))
        return flag, it.value, nf.value, fm.value
