"""ctypes binding of libgemsgpu.so (the C ABI declared in include/gemsgpu.h).

`System` mirrors a GEMS group carrying one interaction group (intergroup,
src/Neighbour.F90:93-208) and one integrator (integrate,
src/Integration.F90:32-49): the setters take the same arguments as the
reference's `interact ... under lj|tb|tersoff` and `evolve v_verlet|ermak`
commands, `interact()` is the reference's interact(), `stepa()/stepb()` are
integration_stepa/b and `dinamica()` is dinamic().  Every call runs on the
GPU through the C ABI; there is no CPU fallback, and importing this module
without the built library raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libgemsgpu.so")

OK = 0
ERRORS = {-1: "ERR_ARG", -2: "ERR_OOM", -3: "ERR_CUDA", -4: "ERR_OVERFLOW", -5: "ERR_LOST",
          -6: "ERR_NAN", -7: "ERR_STATE", -8: "ERR_TIMEOUT", -9: "ERR_NODEV", -10: "ERR_FULL"}
PREC_FP64, PREC_MIXED = 0, 1

# GEMS internal units (src/Constants.F90:101-175)
UI_EV = 1.0e2 * 1.0e2 * 1.6605402e-27 * (1.0 / 1.60219e-19)
EV_UI = 1.0 / UI_EV
KB_UI = 8.617385e-05 * EV_UI

_lib = None
_d, _i, _p, _l = ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class ChpInfo(ctypes.Structure):
    """gemsgpu_chp_info: what a GEMS checkpoint holds beyond the system."""
    _fields_ = [("current", ctypes.c_int32), ("step", ctypes.c_int32), ("nsteps", ctypes.c_int32),
                ("rng", ctypes.c_int32 * 3), ("nframe", ctypes.c_double), ("time", ctypes.c_double),
                ("dm_steps", ctypes.c_double), ("pnframe", ctypes.c_double), ("ptime", ctypes.c_double),
                ("frame", ctypes.c_int32)]


_SIGS = {
    "gemsgpu_version": (ctypes.c_char_p, []),
    "gemsgpu_create": (_i, [_i, _l, _i, ctypes.POINTER(_p)]),
    "gemsgpu_destroy": (_i, [_p]),
    "gemsgpu_last_error": (_i, [_p, ctypes.c_char_p, _i]),
    "gemsgpu_system_create": (_i, [_p, _i, _i, _ip]),
    "gemsgpu_system_destroy": (_i, [_p, _i]),
    "gemsgpu_upload": (_i, [_p, _i, _dp, _dp, _dp, _ip]),
    "gemsgpu_set_positions": (_i, [_p, _i, _dp]),
    "gemsgpu_set_velocities": (_i, [_p, _i, _dp]),
    "gemsgpu_set_accelerations": (_i, [_p, _i, _dp]),
    "gemsgpu_download": (_i, [_p, _i, _dp, _dp, _dp, _dp]),
    "gemsgpu_download_acel": (_i, [_p, _i, _dp]),
    "gemsgpu_set_box": (_i, [_p, _i, _i, _dp, _ip]),
    "gemsgpu_set_skin": (_i, [_p, _i, _d]),
    "gemsgpu_set_list_mode": (_i, [_p, _i, _i]),
    "gemsgpu_set_skin_mode": (_i, [_p, _i, _i]),
    "gemsgpu_set_precision": (_i, [_p, _i, _i]),
    "gemsgpu_set_lj": (_i, [_p, _i, _i, _i, _d, _d, _d, _i, _d]),
    "gemsgpu_set_smatb": (_i, [_p, _i, _i, _i, _d, _d, _d, _d, _d, _d, _d]),
    "gemsgpu_set_tersoff": (_i, [_p, _i, _dp]),
    "gemsgpu_forces": (_i, [_p, _i, _dp, _ip]),
    "gemsgpu_update": (_i, [_p, _i]),
    "gemsgpu_get_list": (_i, [_p, _i, _ip, _ip, _i, _ip]),
    "gemsgpu_get_nupd": (_i, [_p, _i, ctypes.POINTER(_l)]),
    "gemsgpu_set_vv": (_i, [_p, _i, _d]),
    "gemsgpu_set_ermak": (_i, [_p, _i, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_set_ermak_normals": (_i, [_p, _i, _dp]),
    "gemsgpu_set_fire": (_i, [_p, _i, _d, _d]),
    "gemsgpu_set_slj": (_i, [_p, _i, _i, _i, _d, _d, _d]),
    "gemsgpu_set_wca": (_i, [_p, _i, _i, _i, _d, _d]),
    "gemsgpu_set_pred_corr": (_i, [_p, _i, _d]),
    "gemsgpu_set_brownian": (_i, [_p, _i, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_set_scalvel": (_i, [_p, _i, _d, _i, _d]),
    "gemsgpu_set_andersen": (_i, [_p, _i, _d, _d, ctypes.c_uint64]),
    "gemsgpu_clear_thermostat": (_i, [_p, _i]),
    "gemsgpu_set_sm1": (_i, [_p, _i, _i, _i, _d, _d, _d]),
    "gemsgpu_set_feels": (_i, [_p, _i, _i, _i]),
    "gemsgpu_set_virial": (_i, [_p, _i, _i]),
    "gemsgpu_set_lgf": (_i, [_p, _i, _d, _d, _d, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_set_lgf_normals": (_i, [_p, _i, _dp]),
    "gemsgpu_chp_write": (_i, [_p, _i, ctypes.POINTER(ChpInfo), _p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "gemsgpu_chp_read": (_i, [_p, _i, _p, ctypes.c_size_t, ctypes.POINTER(ChpInfo)]),
    "gemsgpu_add_lgf_axis": (_i, [_p, _i, _i, _d, _d, _d, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_set_lkd": (_i, [_p, _i, _d, _d, _d, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_add_ermak_axis": (_i, [_p, _i, _i, _d, _d, _d, ctypes.c_uint64]),
    "gemsgpu_get_box": (_i, [_p, _i, _dp]),
    "gemsgpu_virial": (_i, [_p, _i, _dp]),
    "gemsgpu_pressure": (_i, [_p, _i, _dp]),
    "gemsgpu_step_a": (_i, [_p, _i]),
    "gemsgpu_step_b": (_i, [_p, _i]),
    "gemsgpu_md_steps": (_i, [_p, _i, _i]),
    "gemsgpu_energy": (_i, [_p, _i, _dp, _dp, _dp]),
    "gemsgpu_fmax": (_i, [_p, _i, _dp]),
    "gemsgpu_batch_md_steps": (_i, [_p, _ip, _i, _i]),
    "gemsgpu_batch_fire": (_i, [_p, _ip, _i, _d, _i, _ip]),
    "gemsgpu_batch_energy": (_i, [_p, _ip, _i, _dp, _dp, _dp]),
    "gemsgpu_get_launch_count": (_i, [_p, ctypes.POINTER(_l)]),
    "gemsgpu_get_stream": (_i, [_p, ctypes.POINTER(_p)]),
    "gemsgpu_autotune": (_i, [_p, _i, _i, _ip, _ip, _dp]),
    "gemsgpu_set_lanes": (_i, [_p, _i, _i, _i]),
    "gemsgpu_batch_autotune": (_i, [_p, _ip, _i, _i, _ip, _ip, _dp]),
    "gemsgpu_batch_time_kernels": (_i, [_p, _ip, _i, _i, _dp]),
    "gemsgpu_measure_peaks": (_i, [_i, _dp]),
    "gemsgpu_checkpoint_size": (_i, [_p, _i, ctypes.POINTER(ctypes.c_size_t)]),
    "gemsgpu_checkpoint_save": (_i, [_p, _i, _p, ctypes.c_size_t]),
    "gemsgpu_checkpoint_load": (_i, [_p, _i, _p, ctypes.c_size_t]),
    "gemsgpu_replica_exchange": (_i, [_p, _i, _ip, _dp, _i, ctypes.c_uint64, _dp, _ip]),
    "gemsgpu_lbfgs": (_i, [_p, _i, _i, _d, _d, _i, _ip, _ip, _ip, _dp]),
    "gemsgpu_batch_lbfgs": (_i, [_p, _ip, _i, _i, _d, _d, _i, _ip, _ip, _ip, _dp]),
    "gemsgpu_batch_set_state": (_i, [_p, _ip, _i, _p, _p]),
    "gemsgpu_batch_get_state": (_i, [_p, _ip, _i, _p, _p, _dp, _dp, _dp]),
    "gemsgpu_neb": (_i, [_p, _ip, _i, _ip, _i, _d, _i, _dp, _dp]),
    "gemsgpu_remd_decide": (_i, [_i, _dp, _dp, _i, ctypes.c_uint64, _dp, _ip, _ip]),
    "gemsgpu_retemper": (_i, [_p, _i, _ip, _dp]),
    "gemsgpu_pool_create": (_i, [_p, _i, _l, _l, _i, _i, _i, _i, _i, ctypes.POINTER(_p)]),
    "gemsgpu_pool_destroy": (_i, [_p]),
    "gemsgpu_pool_set": (_i, [_p, _ip, _i]),
    "gemsgpu_pool_run": (_i, [_p, _i]),
    "gemsgpu_server_create": (_i, [_p, _i, _l, _i, _i, _i, _i, ctypes.POINTER(_p)]),
    "gemsgpu_server_destroy": (_i, [_p]),
    "gemsgpu_server_submit": (_i, [_p, _p, ctypes.POINTER(_l)]),
    "gemsgpu_server_step": (_i, [_p, _ip, _ip, _ip]),
    "gemsgpu_server_poll": (_i, [_p, _l, _ip, _dp, _dp, _ip, _dp]),
    "gemsgpu_server_forget": (_i, [_p, _l]),
    "gemsgpu_smatb_forces_noalloc": (_i, [_p, _i, _i, _dp, _ip, _d, _d, _d, _d, _d, _d, _d, _p, _p, _p]),
    "gemsgpu_time_kernels": (_i, [_p, _i, _i, _dp]),
}


def declared_symbols():
    """Every entry point this binding expects the library to export."""
    return sorted(_SIGS)


def lib():
    """Load libgemsgpu.so; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise ImportError("libgemsgpu.so is not built: run __graft_entry__.build() "
                          "(nvcc, sm_100a); there is no CPU fallback")
    L = ctypes.CDLL(LIBPATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class GemsGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


def _ptr(a, ct=ctypes.c_double):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ct))


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if n is not None and a.size != n:
        raise ValueError("expected %d values, got %d" % (n, a.size))
    return a


class Context:
    """One CUDA stream + HBM arena on one device (gemsgpu_ctx)."""

    def __init__(self, device=0, max_atoms=0, max_systems=16):
        h = _p()
        rc = lib().gemsgpu_create(int(device), int(max_atoms), int(max_systems), ctypes.byref(h))
        if rc != OK:
            raise GemsGpuError(rc, "gemsgpu_create failed on device %d" % device)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().gemsgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            lib().gemsgpu_last_error(self.h, buf, 512)
            raise GemsGpuError(rc, buf.value.decode(errors="replace"))

    # batches ---------------------------------------------------------------
    def _ids(self, systems):
        return np.ascontiguousarray([s.sid for s in systems], dtype=np.int32)

    def batch_md_steps(self, systems, nsteps):
        ids = self._ids(systems)
        self.check(lib().gemsgpu_batch_md_steps(self.h, _ptr(ids, ctypes.c_int), len(ids), int(nsteps)))

    def batch_fire(self, systems, fmax, maxit):
        ids = self._ids(systems)
        it = np.zeros(len(ids), dtype=np.int32)
        self.check(lib().gemsgpu_batch_fire(self.h, _ptr(ids, ctypes.c_int), len(ids), float(fmax),
                                            int(maxit), _ptr(it, ctypes.c_int)))
        return it

    def stream_ptr(self):
        """cudaStream_t of this context (int), e.g. for torch.cuda.ExternalStream."""
        v = _p()
        self.check(lib().gemsgpu_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def replica_exchange(self, systems_of_temp, temps, rnd, seed=1, uniforms=None):
        """One parallel-tempering round; returns (systems ordered by temperature, accepted)."""
        ids = self._ids(systems_of_temp)
        t = np.ascontiguousarray(temps, dtype=np.float64)
        u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
        acc = ctypes.c_int()
        self.check(lib().gemsgpu_replica_exchange(self.h, len(ids), _ptr(ids, ctypes.c_int), _ptr(t), int(rnd),
                                                  int(seed), _ptr(u), ctypes.byref(acc)))
        by_id = {s.sid: s for s in systems_of_temp}
        return [by_id[int(k)] for k in ids], acc.value

    def batch_lbfgs(self, systems, m=5, eps=1e-8, xtol=1e-15, itermax=1000):
        """L-BFGS-relax systems together; returns (status, iters, nfun, emin_ev)
        arrays (status 0 converged, 1 iteration limit, -1 line search failed)."""
        ids = self._ids(systems)
        n = len(ids)
        it, nf, stt = (np.zeros(n, dtype=np.int32) for _ in range(3))
        em = np.zeros(n)
        self.check(lib().gemsgpu_batch_lbfgs(self.h, _ptr(ids, ctypes.c_int), n, int(m), float(eps), float(xtol),
                                             int(itermax), _ptr(it, ctypes.c_int), _ptr(nf, ctypes.c_int),
                                             _ptr(stt, ctypes.c_int), _ptr(em)))
        return stt, it, nf, em

    def neb(self, images, fixed, k_ev, iters):
        """Nudged elastic band over image systems (their fixed images set);
        returns (dt in ps, per-image E_pot in eV) and leaves the final band
        in the systems."""
        ids = self._ids(images)
        fx = np.ascontiguousarray(fixed, dtype=np.int32)
        dt = ctypes.c_double()
        e = np.zeros(len(ids))
        self.check(lib().gemsgpu_neb(self.h, _ptr(ids, ctypes.c_int), len(ids), _ptr(fx, ctypes.c_int), len(fx),
                                     float(k_ev), int(iters), ctypes.byref(dt), _ptr(e)))
        return dt.value, e

    @staticmethod
    def _ptrs(arrays, n):
        if arrays is None:
            return None
        out = (ctypes.c_void_p * n)()
        for k, a in enumerate(arrays):
            if a is not None:
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]):
                    raise TypeError("state arrays must be C-contiguous float64 numpy arrays")
                out[k] = a.ctypes.data
        return out

    def batch_set_state(self, systems, pos=None, vel=None):
        """Upload positions and/or velocities (lists of (n, 3) or 3n float64
        arrays, entries may be None) of many systems with one synchronisation."""
        ids = self._ids(systems)
        for arrs in (pos, vel):
            if arrs is not None:
                for s, a in zip(systems, arrs):
                    if a is not None and a.size != 3 * s.n:
                        raise ValueError("system %d needs %d values" % (s.sid, 3 * s.n))
        self.check(lib().gemsgpu_batch_set_state(self.h, _ptr(ids, ctypes.c_int), len(ids),
                                                 self._ptrs(pos, len(ids)), self._ptrs(vel, len(ids))))

    def batch_get_state(self, systems, pos=None, vel=None):
        """Download positions and/or velocities into the given arrays (as in
        batch_set_state) and return (epot_ev, ekin_ev, temp) per system."""
        ids = self._ids(systems)
        n = len(ids)
        for arrs in (pos, vel):
            if arrs is not None:
                for s, a in zip(systems, arrs):
                    if a is not None and a.size != 3 * s.n:
                        raise ValueError("system %d needs %d values" % (s.sid, 3 * s.n))
        ep, ek, t = np.zeros(n), np.zeros(n), np.zeros(n)
        self.check(lib().gemsgpu_batch_get_state(self.h, _ptr(ids, ctypes.c_int), n, self._ptrs(pos, n),
                                                 self._ptrs(vel, n), _ptr(ep), _ptr(ek), _ptr(t)))
        return ep, ek, t

    def retemper(self, systems, temps):
        """New Ermak temperatures, velocities rescaled by sqrt(T_new/T_old)."""
        ids = self._ids(systems)
        t = np.ascontiguousarray(temps, dtype=np.float64)
        self.check(lib().gemsgpu_retemper(self.h, len(ids), _ptr(ids, ctypes.c_int), _ptr(t)))

    def batch_autotune(self, systems, reps=10):
        """One force-kernel launch shape for systems launched together."""
        ids = self._ids(systems)
        k, v, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self.check(lib().gemsgpu_batch_autotune(self.h, _ptr(ids, ctypes.c_int), len(ids), int(reps),
                                                ctypes.byref(k), ctypes.byref(v), ctypes.byref(ms)))
        for s in systems:
            s.tuned = (k.value, v.value, ms.value)
        return k.value, v.value, ms.value

    def batch_time_kernels(self, systems, reps=20):
        """Mean ms of (first force kernel, second, list rebuild) over the set."""
        ids = self._ids(systems)
        out = np.zeros(3)
        self.check(lib().gemsgpu_batch_time_kernels(self.h, _ptr(ids, ctypes.c_int), len(ids), int(reps), _ptr(out)))
        return out

    def launches(self):
        v = ctypes.c_int64()
        self.check(lib().gemsgpu_get_launch_count(self.h, ctypes.byref(v)))
        return v.value

    def batch_energy(self, systems):
        ids = self._ids(systems)
        n = len(ids)
        ep, ek, t = np.zeros(n), np.zeros(n), np.zeros(n)
        self.check(lib().gemsgpu_batch_energy(self.h, _ptr(ids, ctypes.c_int), n, _ptr(ep), _ptr(ek), _ptr(t)))
        return ep, ek, t


_default_ctx = None


def remd_decide(epot_ev, temps, rnd, seed=1, uniforms=None):
    """parallel_tempering2's decision for one round (host arithmetic): returns
    (partner, accepted), partner[k] = the temperature index whose replica
    moves to temps[k]."""
    e = np.ascontiguousarray(epot_ev, dtype=np.float64)
    t = np.ascontiguousarray(temps, dtype=np.float64)
    u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
    n = len(e)
    part = np.zeros(n, dtype=np.int32)
    acc = ctypes.c_int()
    rc = lib().gemsgpu_remd_decide(n, _ptr(e), _ptr(t), int(rnd), int(seed), _ptr(u), _ptr(part, ctypes.c_int),
                                   ctypes.byref(acc))
    if rc != 0:
        raise GemsGpuError("remd_decide: bad arguments (%d)" % rc)
    return part, acc.value


def measure_peaks(device=0):
    """Measured FP32 / FP64 FMA TFLOP/s and MUFU ex2 / rsqrt Gop/s of one device."""
    out = np.zeros(4)
    rc = lib().gemsgpu_measure_peaks(int(device), _ptr(out))
    if rc != 0:
        raise GemsGpuError("measure_peaks failed (%d)" % rc)
    return {"fp32_tflops": float(out[0]), "fp64_tflops": float(out[1]), "ex2_gops": float(out[2]),
            "rsqrt_gops": float(out[3])}


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


class System:
    """A GEMS system on the GPU; setter names follow oracle.System."""

    def __init__(self, pos, mass, types=None, ntypes=1, ctx=None, vel=None):
        self.ctx = ctx or default_context()
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        self.n = pos.shape[0]
        sid = ctypes.c_int()
        self.ctx.check(lib().gemsgpu_system_create(self.ctx.h, self.n, int(ntypes), ctypes.byref(sid)))
        self.sid = sid.value
        self.ntypes = ntypes
        m = _f64(np.broadcast_to(np.asarray(mass, dtype=np.float64), (self.n,)))
        t = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
        v = None if vel is None else _f64(vel, 3 * self.n)
        self._mass = m
        self.ctx.check(lib().gemsgpu_upload(self.ctx.h, self.sid, _ptr(_f64(pos)), _ptr(v), _ptr(m),
                                            _ptr(t, ctypes.c_int)))

    def destroy(self):
        if self.sid is not None:
            self.ctx.check(lib().gemsgpu_system_destroy(self.ctx.h, self.sid))
            self.sid = None

    def _c(self, rc):
        self.ctx.check(rc)

    # state -------------------------------------------------------------------
    def set_pos(self, x):
        self._c(lib().gemsgpu_set_positions(self.ctx.h, self.sid, _ptr(_f64(x, 3 * self.n))))

    def set_vel(self, v):
        self._c(lib().gemsgpu_set_velocities(self.ctx.h, self.sid, _ptr(_f64(v, 3 * self.n))))

    def set_acel(self, a):
        self._c(lib().gemsgpu_set_accelerations(self.ctx.h, self.sid, _ptr(_f64(a, 3 * self.n))))

    def _down(self, which):
        out = np.empty(3 * self.n if which != 3 else self.n, dtype=np.float64)
        args = [None, None, None, None]
        args[which] = _ptr(out)
        self._c(lib().gemsgpu_download(self.ctx.h, self.sid, *args))
        return out.reshape(self.n, 3) if which != 3 else out

    @property
    def pos(self):
        return self._down(0)

    @property
    def vel(self):
        return self._down(1)

    @property
    def force(self):
        return self._down(2)

    @property
    def epot_atoms(self):
        return self._down(3)

    @property
    def acel(self):
        out = np.empty(3 * self.n, dtype=np.float64)
        self._c(lib().gemsgpu_download_acel(self.ctx.h, self.sid, _ptr(out)))
        return out.reshape(self.n, 3)

    # setup -------------------------------------------------------------------
    def set_box(self, L=None, pbc=(True, True, True)):
        if L is None:
            self._c(lib().gemsgpu_set_box(self.ctx.h, self.sid, 0, None, None))
            return
        Lb = _f64(L, 3)
        pb = np.asarray([1 if b else 0 for b in pbc], dtype=np.int32)
        self._c(lib().gemsgpu_set_box(self.ctx.h, self.sid, 1, _ptr(Lb), _ptr(pb, ctypes.c_int)))

    def set_skin(self, skin):
        self._c(lib().gemsgpu_set_skin(self.ctx.h, self.sid, float(skin)))

    def set_skin_mode(self, mic):
        """mic=False: the reference's raw-displacement skin test."""
        self._c(lib().gemsgpu_set_skin_mode(self.ctx.h, self.sid, 1 if mic else 0))

    def set_half(self, half):
        self._c(lib().gemsgpu_set_list_mode(self.ctx.h, self.sid, 1 if half else 0))

    def set_precision(self, prec):
        self._c(lib().gemsgpu_set_precision(self.ctx.h, self.sid, int(prec)))

    def set_lj(self, e, s, rc, ti=0, tj=0, shifted_force=False, eshift=0.0):
        self._c(lib().gemsgpu_set_lj(self.ctx.h, self.sid, ti, tj, e, s, rc, 1 if shifted_force else 0, eshift))

    def set_slj(self, e, sg, rs, ti=0, tj=0):
        """slj_set: LJ core to rs, polynomial tail to the derived cut-off."""
        self._c(lib().gemsgpu_set_slj(self.ctx.h, self.sid, ti, tj, float(e), float(sg), float(rs)))

    def set_wca(self, e, s, ti=0, tj=0):
        """wca_set: LJ cut at its minimum and shifted up by e."""
        self._c(lib().gemsgpu_set_wca(self.ctx.h, self.sid, ti, tj, float(e), float(s)))

    def set_sm1(self, r1, r2, e, ti=0, tj=0):
        """sm1_set: smooth step of depth e (eV) from r1 to r2."""
        self._c(lib().gemsgpu_set_sm1(self.ctx.h, self.sid, ti, tj, float(r1), float(r2), float(e)))

    def set_feels(self, ti, tj):
        """`interact g1 feels g2`: the pair (ti, tj) acts on type ti only."""
        self._c(lib().gemsgpu_set_feels(self.ctx.h, self.sid, int(ti), int(tj)))

    def set_virial(self, on=True):
        self._c(lib().gemsgpu_set_virial(self.ctx.h, self.sid, 1 if on else 0))

    def set_smatb(self, A, xi, p, q, r0, rci, rce, ti=0, tj=0):
        self._c(lib().gemsgpu_set_smatb(self.ctx.h, self.sid, ti, tj, A, xi, p, q, r0, rci, rce))

    def set_tersoff(self, prm):
        a = _f64(prm, 12)
        self._c(lib().gemsgpu_set_tersoff(self.ctx.h, self.sid, _ptr(a)))

    # compute -----------------------------------------------------------------
    def interact(self):
        """interact(): forces, per-atom energies; returns Epot (internal units)."""
        e = ctypes.c_double()
        self._c(lib().gemsgpu_forces(self.ctx.h, self.sid, ctypes.byref(e), None))
        return e.value

    def update(self):
        self._c(lib().gemsgpu_update(self.ctx.h, self.sid))

    @property
    def nupd(self):
        v = ctypes.c_int64()
        self._c(lib().gemsgpu_get_nupd(self.ctx.h, self.sid, ctypes.byref(v)))
        return v.value

    def neighbour_list(self):
        need = ctypes.c_int()
        nn = np.empty(self.n, dtype=np.int32)
        self._c(lib().gemsgpu_get_list(self.ctx.h, self.sid, _ptr(nn, ctypes.c_int), None, 0, ctypes.byref(need)))
        cap = max(need.value, 1)
        lst = np.empty(cap * self.n, dtype=np.int32)
        self._c(lib().gemsgpu_get_list(self.ctx.h, self.sid, _ptr(nn, ctypes.c_int), _ptr(lst, ctypes.c_int),
                                       cap, ctypes.byref(need)))
        return nn, lst.reshape(cap, self.n)

    def pair_set(self):
        nn, lst = self.neighbour_list()
        i_idx = np.repeat(np.arange(self.n, dtype=np.int64), nn)
        j_idx = np.concatenate([lst[:c, i].astype(np.int64) for i, c in enumerate(nn)]) if self.n else np.zeros(0, np.int64)
        return np.sort(i_idx * self.n + j_idx)

    # integrators -------------------------------------------------------------
    def set_vv(self, dt):
        self._axes = []
        self._c(lib().gemsgpu_set_vv(self.ctx.h, self.sid, float(dt)))

    def set_pred_corr(self, dt):
        """`evolve pred_corr_5`: the fifth-order Nordsieck predictor-corrector."""
        self._axes = []
        self._c(lib().gemsgpu_set_pred_corr(self.ctx.h, self.sid, float(dt)))

    def set_ermak(self, dt, gama, temp, seed=12345):
        self._axes = []
        self._c(lib().gemsgpu_set_ermak(self.ctx.h, self.sid, float(dt), float(gama), float(temp), int(seed)))

    def set_brownian(self, dt, temp, gama, seed=12345):
        """`evolve brownian temp gama`: overdamped Langevin (cbrownian)."""
        self._axes = []
        self._c(lib().gemsgpu_set_brownian(self.ctx.h, self.sid, float(dt), float(temp), float(gama), int(seed)))

    def set_scalvel(self, temp, steps, upto=None):
        """`evolve scalvel temp steps` (scalvel_after with upto), run after
        the integrator's step b."""
        self._c(lib().gemsgpu_set_scalvel(self.ctx.h, self.sid, float(temp), int(steps),
                                          -1.0 if upto is None else float(upto)))

    def set_andersen(self, temp, nu=20.0, seed=4242):
        """`evolve andersen temp nu`, run after the integrator's step b."""
        self._c(lib().gemsgpu_set_andersen(self.ctx.h, self.sid, float(temp), float(nu), int(seed)))

    def clear_thermostat(self):
        self._c(lib().gemsgpu_clear_thermostat(self.ctx.h, self.sid))

    def set_ermak_normals(self, nrm):
        a = None if nrm is None else _f64(nrm, 6 * self.n)
        self._c(lib().gemsgpu_set_ermak_normals(self.ctx.h, self.sid, _ptr(a)))

    def set_fire(self, dt0, dtmax):
        self._axes = []
        self._c(lib().gemsgpu_set_fire(self.ctx.h, self.sid, float(dt0), float(dtmax)))

    def set_lgf(self, dt, temp, press_atm, pgama0, pgamav, pmass, seed=12345):
        """set_lgf (`evolve piston_lgf xyz*`): G-JF constant pressure and
        temperature; pressure in atm, frictions in 1/ps."""
        self._axes = []
        self._c(lib().gemsgpu_set_lgf(self.ctx.h, self.sid, float(dt), float(temp), float(press_atm),
                                      float(pgama0), float(pgamav), float(pmass), int(seed)))

    def set_lkd(self, dt, temp, press_atm, pgama0, pgamav, pmass, seed=12345):
        """set_lkd (`evolve piston_lkd`): the Langevin piston of Kolb & Dunweg."""
        self._axes = ["lkd"]
        self._c(lib().gemsgpu_set_lkd(self.ctx.h, self.sid, float(dt), float(temp), float(press_atm),
                                      float(pgama0), float(pgamav), float(pmass), int(seed)))

    def add_lgf_axis(self, axis, dt, temp, press_atm, pgama0, pgamav, pmass, seed=12345):
        """`evolve piston_lgf x|y|z`: a G-JF piston on one box length."""
        if getattr(self, "_axes", []) == ["lkd"]:
            self._axes = []
        self._c(lib().gemsgpu_add_lgf_axis(self.ctx.h, self.sid, int(axis), float(dt), float(temp),
                                           float(press_atm), float(pgama0), float(pgamav), float(pmass),
                                           int(seed)))
        self._axes = getattr(self, "_axes", []) + ["lgf"]

    def add_ermak_axis(self, axis, dt, gama, temp, seed=12345):
        """`evolve ermak_x|y|z`: Ermak dynamics of one coordinate."""
        if getattr(self, "_axes", []) == ["lkd"]:
            self._axes = []
        self._c(lib().gemsgpu_add_ermak_axis(self.ctx.h, self.sid, int(axis), float(dt), float(gama),
                                             float(temp), int(seed)))
        self._axes = getattr(self, "_axes", []) + ["ermak"]

    def set_lgf_normals(self, nrm):
        """Next step's normal pairs in the order the reference draws them:
        isotropic piston -- the piston's pair, then a pair per atom
        coordinate (2 + 6 n values); per-coordinate integrators -- for each
        in order, a piston's pair and a pair per atom, or a pair per atom.
        None returns to the device stream."""
        axes = getattr(self, "_axes", [])
        if axes == ["lkd"]:
            pairs = 6 * self.n + 2
        else:
            pairs = sum(1 + self.n if a == "lgf" else self.n for a in axes) if axes else 1 + 3 * self.n
        a = None if nrm is None else _f64(nrm, 2 * pairs)
        self._c(lib().gemsgpu_set_lgf_normals(self.ctx.h, self.sid, _ptr(a)))

    def box_now(self):
        L = np.empty(3, dtype=np.float64)
        self._c(lib().gemsgpu_get_box(self.ctx.h, self.sid, _ptr(L)))
        return L

    def virial_ev(self):
        """Pair virial of the last force evaluation (eV, xx xy xz yx ... zz)."""
        out = np.empty(9, dtype=np.float64)
        self._c(lib().gemsgpu_virial(self.ctx.h, self.sid, _ptr(out)))
        return out

    def pressure_atm(self):
        """Pressure tensor (sum m v v + W) / V in atm, row-major."""
        out = np.empty(9, dtype=np.float64)
        self._c(lib().gemsgpu_pressure(self.ctx.h, self.sid, _ptr(out)))
        return out

    def stepa(self):
        self._c(lib().gemsgpu_step_a(self.ctx.h, self.sid))

    def stepb(self):
        self._c(lib().gemsgpu_step_b(self.ctx.h, self.sid))

    def md_steps(self, n):
        self._c(lib().gemsgpu_md_steps(self.ctx.h, self.sid, int(n)))

    def energy(self):
        """(Epot eV, Ekin eV with CM removed, T K)."""
        ep, ek, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._c(lib().gemsgpu_energy(self.ctx.h, self.sid, ctypes.byref(ep), ctypes.byref(ek), ctypes.byref(t)))
        return ep.value, ek.value, t.value

    def kin(self):
        _, ek, t = self.energy()
        return ek * EV_UI, t

    def epot_sum(self):
        return self.energy()[0] * EV_UI

    def autotune(self, reps=10):
        """Pick the fastest force-kernel launch shape; returns (lanes, variant, ms)."""
        k, v, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._c(lib().gemsgpu_autotune(self.ctx.h, self.sid, int(reps), ctypes.byref(k), ctypes.byref(v),
                                       ctypes.byref(ms)))
        return k.value, v.value, ms.value

    def set_lanes(self, lanes, variant=1):
        self._c(lib().gemsgpu_set_lanes(self.ctx.h, self.sid, int(lanes), int(variant)))

    def time_kernels(self, reps=20):
        """Mean ms of (first force kernel, second force kernel, list rebuild)."""
        out = np.zeros(3)
        self._c(lib().gemsgpu_time_kernels(self.ctx.h, self.sid, int(reps), _ptr(out)))
        return out

    def checkpoint(self):
        """write_chp: the system's resumable state as bytes."""
        n = ctypes.c_size_t()
        self._c(lib().gemsgpu_checkpoint_size(self.ctx.h, self.sid, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._c(lib().gemsgpu_checkpoint_save(self.ctx.h, self.sid, buf, n.value))
        return buf.raw

    def restore(self, data):
        """read_chp: resume from checkpoint bytes (the next interact rebuilds the list)."""
        buf = ctypes.create_string_buffer(data, len(data))
        self._c(lib().gemsgpu_checkpoint_load(self.ctx.h, self.sid, buf, len(data)))

    def write_gems_chp(self, current=1, step=0, nsteps=0, rng=(0, 0, 0), **frame):
        """write_chp: GEMS's checkpoint file as bytes (rng = lcg idum, iy, ix;
        frame: nframe, time, dm_steps, pnframe, ptime, frame)."""
        info = ChpInfo(current, step, nsteps, (ctypes.c_int32 * 3)(*rng), frame.get("nframe", 0.0),
                       frame.get("time", 0.0), frame.get("dm_steps", 0.0), frame.get("pnframe", 0.0),
                       frame.get("ptime", 0.0), frame.get("frame", 0))
        n = ctypes.c_size_t()
        self._c(lib().gemsgpu_chp_write(self.ctx.h, self.sid, ctypes.byref(info), None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._c(lib().gemsgpu_chp_write(self.ctx.h, self.sid, ctypes.byref(info), buf, n.value, ctypes.byref(n)))
        return buf.raw[:n.value]

    def read_gems_chp(self, data):
        """read_chp: resume from GEMS checkpoint bytes; returns the file's
        counters and generator state as a dict."""
        buf = ctypes.create_string_buffer(data, len(data))
        info = ChpInfo()
        self._c(lib().gemsgpu_chp_read(self.ctx.h, self.sid, buf, len(data), ctypes.byref(info)))
        return {"current": info.current, "step": info.step, "nsteps": info.nsteps, "rng": tuple(info.rng),
                "nframe": info.nframe, "time": info.time, "dm_steps": info.dm_steps, "pnframe": info.pnframe,
                "ptime": info.ptime, "frame": info.frame}

    def lbfgs(self, m=5, eps=1e-8, xtol=1e-15, itermax=1000):
        """lbfgs_minimizator: minimise in place; returns (status, iterations,
        function evaluations, E_pot in eV) -- status 0 converged, 1 iteration
        limit, -1 line search failed."""
        it, nf, st, em = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._c(lib().gemsgpu_lbfgs(self.ctx.h, self.sid, int(m), float(eps), float(xtol), int(itermax),
                                    ctypes.byref(it), ctypes.byref(nf), ctypes.byref(st), ctypes.byref(em)))
        return st.value, it.value, nf.value, em.value

    def fmax(self):
        v = ctypes.c_double()
        self._c(lib().gemsgpu_fmax(self.ctx.h, self.sid, ctypes.byref(v)))
        return v.value

    def dinamica(self, nsteps, each):
        """dinamic(): interact once, then nsteps on the device; every `each`
        steps one row (Epot, Ekin, Etot in eV, T in K)."""
        self.interact()
        rows = []
        done = 0
        while done < nsteps:
            k = min(each, nsteps - done) if each > 0 else nsteps
            self.md_steps(k)
            done += k
            if each > 0 and done % each == 0:
                ep, ek, t = self.energy()
                rows.append([ep, ek, ep + ek, t])
        return np.array(rows).reshape(-1, 4)


FF_LJ, FF_SMATB, FF_TERSOFF = 1, 2, 3
JOB_FIRE, JOB_MD = 0, 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class Pool:
    """A fixed-capacity set of systems advanced through one captured graph."""

    def __init__(self, ctx, max_systems, max_atoms, max_cells=1, ff=FF_SMATB, prec=PREC_MIXED, lanes=8,
                 variant=1, chunk=50):
        self.ctx = ctx
        h = _p()
        ctx.check(lib().gemsgpu_pool_create(ctx.h, int(max_systems), int(max_atoms), int(max_cells), int(ff),
                                            int(prec), int(lanes), int(variant), int(chunk), ctypes.byref(h)))
        self.h = h

    def set(self, systems):
        ids = np.ascontiguousarray([s.sid for s in systems], dtype=np.int32)
        self.ctx.check(lib().gemsgpu_pool_set(self.h, _ptr(ids, ctypes.c_int), len(ids)))

    def run(self, nchunks=1):
        self.ctx.check(lib().gemsgpu_pool_run(self.h, int(nchunks)))

    def close(self):
        if getattr(self, "h", None):
            lib().gemsgpu_pool_destroy(self.h)
            self.h = None


class _Job(ctypes.Structure):
    _fields_ = [("natoms", ctypes.c_int), ("pos", ctypes.POINTER(ctypes.c_double)), ("mass", ctypes.c_double),
                ("smatb", ctypes.c_double * 7), ("kind", ctypes.c_int), ("steps", ctypes.c_int),
                ("dt", ctypes.c_double), ("temp", ctypes.c_double), ("gamma", ctypes.c_double),
                ("fmax", ctypes.c_double), ("seed", ctypes.c_uint64)]


class Server:
    """The serving loop (gemsgpu_server_*): submit jobs, step, poll."""

    def __init__(self, ctx, max_jobs, max_atoms, prec=PREC_MIXED, lanes=4, variant=1, chunk=50):
        self.ctx = ctx
        h = _p()
        ctx.check(lib().gemsgpu_server_create(ctx.h, int(max_jobs), int(max_atoms), int(prec), int(lanes),
                                              int(variant), int(chunk), ctypes.byref(h)))
        self.h = h
        self.sizes = {}

    def submit(self, pos, mass, smatb, kind, steps, dt=0.002, temp=300.0, gamma=1.0, fmax=1e-3, seed=1):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        j = _Job()
        j.natoms = p.size // 3
        j.pos = _ptr(p)
        j.mass = float(mass)
        for k in range(7):
            j.smatb[k] = float(smatb[k])
        j.kind, j.steps, j.dt, j.temp, j.gamma, j.fmax, j.seed = (int(kind), int(steps), float(dt), float(temp),
                                                                  float(gamma), float(fmax), int(seed))
        jid = ctypes.c_int64()
        self.ctx.check(lib().gemsgpu_server_submit(self.h, ctypes.byref(j), ctypes.byref(jid)))
        self.sizes[jid.value] = j.natoms
        return jid.value

    def step(self):
        r, q, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.ctx.check(lib().gemsgpu_server_step(self.h, ctypes.byref(r), ctypes.byref(q), ctypes.byref(f)))
        return r.value, q.value, f.value

    def poll(self, jid, want_pos=False):
        st, ep, fm, it = ctypes.c_int(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        pos = np.zeros(3 * self.sizes[jid]) if want_pos else None
        self.ctx.check(lib().gemsgpu_server_poll(self.h, int(jid), ctypes.byref(st), ctypes.byref(ep),
                                                 ctypes.byref(fm), ctypes.byref(it), _ptr(pos)))
        out = {"state": st.value, "epot_ev": ep.value, "fmax_ev": fm.value, "iters": it.value}
        if want_pos:
            out["pos"] = pos.reshape(-1, 3)
        return out

    def forget(self, jid):
        self.ctx.check(lib().gemsgpu_server_forget(self.h, int(jid)))

    def close(self):
        if getattr(self, "h", None):
            lib().gemsgpu_server_destroy(self.h)
            self.h = None
