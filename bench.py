"""Benchmark of the GEMS force/neighbour path on B200.

Workload (default): 32000-atom SMA-TB Au bulk (fcc 20^3, a=4.078 A, periodic,
seeded N(0, 0.02 A) displacements), Ermak Langevin 300 K, gamma=1/ps, dt=2 fs.
Metric: atom-steps/s (one atom-step = one force evaluation + one integrator
update for one atom, neighbour rebuilds amortised in).

One bench step = one block of --block MD steps (default 100) run on the
device through the C ABI (gemsgpu_batch_md_steps).  The L2 is flushed
(a 256 MiB write) between timed blocks, outside the timed events.

Arms measured in one run:
  fp64   : the plain FP64 drop-in kernels, one system;
  mixed  : FP32 pair math with FP64 accumulation, one system;
  batched: the mixed kernels over --replicas independent 32k-atom replicas
           (different displacement / noise seeds) packed into one launch.
  batched_fp64: the same replicas in the plain FP64 kernels (splits the
           headline into batching and precision).
`value` is the batched arm; every arm is reported.  `e2e` runs the batched
arm through the C ABI with host buffers: each block uploads positions and
velocities from pinned memory and reads positions, velocities and energies
back.  `e2e_dropin_per_step` times the per-step drop-in path instead: a GEMS
build that keeps its host integrator and calls gemsgpu_set_positions,
gemsgpu_forces and gemsgpu_download every MD step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s on 1 B200 (FP32+FP64-acc vs plain FP64); serve p50/p99 latency"
UNIT = "atom-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--block", type=int, default=100, help="MD steps per bench step")
    ap.add_argument("--replicas", type=int, default=8)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--arms", default="fp64,mixed,batched",
                    help="comma list of arms to run (profiling; 'rebuild' times the batch's list "
                         "rebuild alone); the full line needs fp64,mixed,batched")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--therm-steps", type=int, default=None,
                    help="reference arm: untimed Ermak steps before timing (default: the GPU arms' %d)"
                         % THERM_STEPS)
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5", "next"],
                    help="c2 (default, the headline line) or one of the other configurations")
    ap.add_argument("--serve-seconds", type=float, default=20.0,
                    help="c4: length of the Poisson arrival window (the full configuration is 120 s)")
    ap.add_argument("--tune", default=None,
                    help="lanes,variant for every mixed system instead of the autotuner (profiling)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value, dist, device=None):
    """The largest value over all ranks (timings are the slowest rank's)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.mark = 0
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi takes a while to print its first line: wait for it, so
        # that the samples kept (from here on) cover the timed region
        t_end = time.time() + 5.0
        while not self.samples and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.01)
        self.mark = len(self.samples)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            # one more sample at the end of the timed region (100 ms period)
            n = len(self.samples)
            t_end = time.time() + 0.3
            while len(self.samples) == n and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        self.samples = self.samples[self.mark:] or self.samples[-1:]
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- workload
def c2_replica(seed):
    from gems_b200 import workloads as W
    return W.smatb_bulk(seed=seed)


FIXED_TUNE = None


# The C2 lattice starts at 0 K and the thermostat takes a few ps to bring it
# to 300 K; a cold crystal runs ~30 % faster (its lists hardly ever rebuild
# and stay distance-sorted), so every arm is thermalised before it is tuned
# and timed: 2000 steps = 4 ps = four relaxation times 1/gamma.
THERM_STEPS = 2000


def make_system(gems, ctx, w, prec, seed, tune=None, therm=THERM_STEPS):
    """One C2 system, thermalised by `therm` untimed steps; `tune` copies a
    launch shape, else the autotuner picks (on the thermalised state)."""
    s = gems.System(w["pos"], w["mass"], ctx=ctx)
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    s.set_skin(w["skin"])
    s.set_precision(prec)
    s.set_ermak(w["dt"], w["gamma"], w["temp"], seed=seed)
    s.interact()
    if tune is None and FIXED_TUNE is not None:
        tune = FIXED_TUNE
    if tune is not None:
        s.set_lanes(tune[0], tune[1])
        s.tuned = tune
    if therm:
        s.md_steps(therm)
    if tune is None:
        s.tuned = s.autotune(10)
    return s


def smatb_pair_stats(s, L, rci, rce):
    """List entries, pairs with r <= rci and pairs with rci < r <= rce of one
    periodic system at its current positions (minimum image)."""
    nn, lst = s.neighbour_list()
    x = s.pos
    i = np.repeat(np.arange(s.n), nn)
    j = np.concatenate([lst[:c, a] for a, c in enumerate(nn)]).astype(np.int64)
    d = x[j] - x[i]
    Lv = np.asarray(L, dtype=np.float64)
    d -= Lv * np.round(d / Lv)
    r = np.sqrt((d * d).sum(1))
    return {"entries": int(nn.sum()), "inner": int((r <= rci).sum()),
            "tail": int(((r > rci) & (r <= rce)).sum())}


def smatb_compute_counts(st):
    """Algorithmic FP32 flops (FMA = 2) and MUFU operations of the two mixed
    SMA-TB passes for the pair statistics `st`:
      every list entry: pair vector and r^2 (8 flops);
      density, r <= rci: rsqrt + Newton (4), exp argument and scale (3), sum (1); 2 MUFU
      density, tail:      rsqrt + Newton (4), quintic and square (8), sum (1);    1 MUFU
      force,   r <= rci: rsqrt + Newton (4), eband sum (1), two exps and factor (8),
                         force and energy sums (9);                                3 MUFU
      force,   tail:      rsqrt + Newton (4), eband sum (1), three polynomials and
                         factor (34), force and energy sums (9);                   1 MUFU"""
    e, a, b = st["entries"], st["inner"], st["tail"]
    rho = {"flops": 8 * e + 8 * a + 13 * b, "mufu": 2 * a + b}
    force = {"flops": 8 * e + 22 * a + 48 * b, "mufu": 3 * a + b}
    return rho, force


def compute_roof(counts, bytes_, ms, peaks, hbm):
    """Time each roof allows for one launch, and the fraction of the binding one."""
    t = {"hbm_us": bytes_ / (hbm * 1e9) * 1e6,
         "fp32_us": counts["flops"] / (peaks["fp32_tflops"] * 1e12) * 1e6,
         "mufu_us": counts["mufu"] / (peaks["ex2_gops"] * 1e9) * 1e6}
    bind = max(t, key=t.get)
    return {"flops_per_launch": counts["flops"], "mufu_per_launch": counts["mufu"],
            "roof_times_us": t, "binding": bind.replace("_us", ""), "measured_us": ms * 1e3,
            "frac_of_binding_roof": t[bind] / (ms * 1e3)}


def timed_blocks(ctx, torch, systems, block, steps, warmup, flush, ext_stream):
    """Run warmup + steps blocks of `block` MD steps; returns (ms list, launches)."""
    for _ in range(warmup):
        ctx.batch_md_steps(systems, block)
    torch.cuda.synchronize()
    times = []
    l0 = ctx.launches()
    for _ in range(steps):
        flush.add_(1.0)  # > L2, on torch's stream
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext_stream)
        ctx.batch_md_steps(systems, block)
        e1.record(ext_stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times, ctx.launches() - l0


def timed_e2e(ctx, torch, systems, block, steps, warmup, flush, ext_stream):
    """Same blocks through the C ABI with host buffers (pinned), H2D of
    positions + velocities and D2H of positions, velocities and energies inside
    the timed region."""
    n = sum(s.n for s in systems)
    host = []
    for s in systems:
        p = torch.empty(3 * s.n, dtype=torch.float64).pin_memory()
        v = torch.empty(3 * s.n, dtype=torch.float64).pin_memory()
        p.numpy()[:] = s.pos.ravel()
        v.numpy()[:] = s.vel.ravel()
        host.append((p, v))

    pos_h = [p.numpy() for p, _ in host]
    vel_h = [v.numpy() for _, v in host]

    def one():
        ctx.batch_set_state(systems, pos_h, vel_h)
        ctx.batch_md_steps(systems, block)
        return ctx.batch_get_state(systems, pos_h, vel_h)

    for _ in range(warmup):
        one()
    times = []
    for _ in range(steps):
        flush.add_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext_stream)
        one()
        e1.record(ext_stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    h2d = 2 * 24 * n
    d2h = 2 * 24 * n + 24 * len(systems)
    return times, h2d, d2h


def ermak_consts(dt, gamma, temp):
    """set_ermak (src/Integration.F90:909-961) for the host-side integrator
    of the per-step drop-in arm."""
    from gems_b200 import workloads as W
    c0 = np.exp(-gamma * dt)
    c1 = (1.0 - c0) / gamma
    c2 = (1.0 - c1 / dt) / gamma
    sdr = np.sqrt(dt / gamma * (2.0 - (3.0 - 4.0 * c0 + c0 * c0) / (gamma * dt)))
    sdv = np.sqrt(1.0 - c0 * c0)
    crv1 = (1.0 - c0) ** 2 / (gamma * sdr * sdv)
    crv2 = np.sqrt(1.0 - crv1 * crv1)
    return dict(dt=dt, c0=c0, c1=c1, c2=c2, sdr=sdr, sdv=sdv, crv1=crv1, crv2=crv2,
                skt=np.sqrt(W.KB_UI * temp))


def timed_dropin(gems, torch, ctx, ext, s, w, steps, warmup=5):
    """The per-step drop-in path: a GEMS build that keeps its own (host)
    integrator and swaps only the force field for the GPU one, through the
    Fortran interact() shim.  Every MD step: ermak_a on the host, upload of
    the positions (gemsgpu_set_positions), gemsgpu_forces, download of
    forces and per-atom energies (gemsgpu_download), ermak_b on the host
    (src/Integration.F90:963-1031, in numpy).  Timed with CUDA events on the
    library's stream around `steps` MD steps, host work included."""
    import ctypes
    lib = gems.lib()
    n = s.n
    K = ermak_consts(w["dt"], w["gamma"], w["temp"])
    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    x, v, a, f, e = pin((n, 3)), pin((n, 3)), pin((n, 3)), pin((n, 3)), pin((n,))
    x[:] = s.pos
    v[:] = s.vel
    a[:] = s.acel
    m = float(w["mass"])
    osm = 1.0 / np.sqrt(m)
    L = np.asarray(w["L"], dtype=np.float64)
    rng = np.random.default_rng(17)
    ep = ctypes.c_double()
    P = lambda arr: arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    px, pf, pe = P(x), P(f), P(e)
    r = np.empty((2, n, 3))
    vel_v = np.empty((n, 3))

    def step():
        rng.standard_normal(out=r)
        fl = K["skt"] * osm
        np.multiply(r[0], fl * K["sdr"], out=f)            # pos_v (f is free until the download)
        x[:] += K["c1"] * v + (K["c2"] * K["dt"]) * a + f
        np.subtract(x, L * np.floor(x / L), out=x)            # do_pbc
        np.multiply(fl * K["sdv"], K["crv1"] * r[0] + K["crv2"] * r[1], out=vel_v)
        ctx.check(lib.gemsgpu_set_positions(ctx.h, s.sid, px))
        ctx.check(lib.gemsgpu_forces(ctx.h, s.sid, ctypes.byref(ep), None))
        ctx.check(lib.gemsgpu_download(ctx.h, s.sid, None, None, pf, pe))
        v[:] = K["c0"] * v + (K["c1"] - K["c2"]) * a + (K["c2"] / m) * f + vel_v
        np.multiply(f, 1.0 / m, out=a)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(ext)
    for _ in range(steps):
        step()
    e1.record(ext)
    e1.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    return {"value": n * steps / (ms * 1e-3), "unit": UNIT, "md_steps": steps, "atoms": n,
            "ms_per_md_step": ms / steps, "wall_ms_per_md_step": 1e3 * wall / steps,
            "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 32 * n,
            "path": "per MD step: host ermak_a, gemsgpu_set_positions, gemsgpu_forces, gemsgpu_download "
                    "(forces, energies), host ermak_b"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_baseline(seconds, state=None):
    """The FP64 OpenMP restatement (oracle port) on all host cores: C2 sample,
    from the thermalised state (pos, vel, acel) the GPU arms start from."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    w = c2_replica(2)
    s = O.System(w["pos"], w["mass"])
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    s.set_skin(w["skin"])
    s.set_ermak(w["dt"], w["gamma"], w["temp"], O.Rng(123456))
    if state is not None:
        s.set_pos(state[0])
        s.set_vel(state[1])
        s.set_acel(state[2])
    s.interact()
    t0 = time.perf_counter()
    steps = 0
    while True:
        s.stepa()
        s.interact()
        s.stepb()
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 3:
            break
    return {"value": s.n * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d MD steps of the 32000-atom SMA-TB Ermak workload from the thermalised 300 K state "
                      "(FP64 OpenMP restatement)" % steps}


def _cpu_steps(s, seconds):
    """Step an oracle system (stepa, interact, stepb) for about `seconds`."""
    s.interact()
    t0 = time.perf_counter()
    steps = 0
    while True:
        s.stepa()
        s.interact()
        s.stepb()
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 3:
            return steps, el


def cpu_baseline_c1(seconds):
    from oracle import oracle as O
    from gems_b200 import workloads as W
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    w = W.lj_fluid()
    s = O.System(w["pos"], 1.0)
    s.set_vel(w["vel"])
    s.set_box(w["L"], (True, True, True))
    e, sg, rc, sh = w["lj"]
    s.set_lj(e, sg, rc, eshift=sh)
    s.set_skin(w["skin"])
    s.set_vv(w["dt"])
    steps, el = _cpu_steps(s, seconds)
    return {"value": s.n * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d VV steps of the 4000-atom LJ fluid (FP64 OpenMP restatement)" % steps}


def cpu_baseline_c5(seconds):
    from oracle import oracle as O
    from gems_b200 import workloads as W
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    w = W.tersoff_si()
    s = O.System(w["pos"], w["mass"])
    s.set_vel(w["vel"])
    s.set_box(w["L"], (True, True, True))
    s.set_tersoff(w["tersoff"])
    s.set_skin(w["skin"])
    s.set_vv(w["dt"])
    steps, el = _cpu_steps(s, seconds)
    return {"value": s.n * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d VV steps of the 1,000,000-atom Tersoff Si crystal (FP64 OpenMP restatement)" % steps}


def cpu_baseline_c3(seconds):
    """FIRE relaxations of the batch's first clusters, one after another."""
    from oracle import oracle as O
    from gems_b200 import workloads as W
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    sm, m = W.SMATB["Au"], W.MASS["Au"]
    clusters = W.batched_clusters()
    t0 = time.perf_counter()
    work, done = 0.0, 0
    for p in clusters[:64]:
        s = O.System(p, m)
        s.set_smatb(*sm)
        s.set_fire(0.002, 0.02)
        it, _ = s.fire_relax(1e-3, 5000)
        work += it * s.n
        done += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    return {"value": work / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "FIRE to 1e-3 eV/A of the first %d clusters of the batch, one after another "
                      "(FP64 OpenMP restatement)" % done}


def run_reference(args):
    """The reference's CPU path (the FP64 OpenMP restatement: no Fortran
    compiler exists to build the reference itself), on this config."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    w = c2_replica(2)
    s = O.System(w["pos"], w["mass"])
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    s.set_skin(w["skin"])
    s.set_ermak(w["dt"], w["gamma"], w["temp"], O.Rng(123456))
    s.interact()
    # the same start as the GPU arms: thermalised at 300 K, here by the CPU
    # restatement's own Ermak steps (untimed)
    nth = THERM_STEPS if args.therm_steps is None else max(0, args.therm_steps)
    t_th = time.perf_counter()
    for _ in range(nth):
        s.stepa()
        s.interact()
        s.stepb()
    t_th = time.perf_counter() - t_th
    per = max(1, min(args.block, 5))   # bounded sample per bench step

    def blk():
        for _ in range(per):
            s.stepa()
            s.interact()
            s.stepb()

    for _ in range(args.warmup):
        blk()
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        blk()
        ts.append(time.perf_counter() - t0)
    tot = sum(ts)
    val = s.n * per * args.steps / tot
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "smatb_au_bulk_32000 (fcc 20^3, Ermak 300 K, dt 2 fs)",
                       "md_steps_per_bench_step": per, "parallelism": "openmp",
                       "start": "thermalised: %d untimed Ermak steps (%.3g ps) from the 0 K lattice, "
                                "by the CPU restatement itself (%.0f s)" % (nth, nth * w["dt"], t_th),
                       "skin_test": "the reference's (raw displacements, src/Neighbour.F90:1320)"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d blocks of %d MD steps, 32000 atoms, from the thermalised "
                                       "300 K state" % (args.steps, per)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- other configs
def _line(metric, value, unit, args, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
         "data": "synthetic", "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def _time_md(ctx, torch, systems, block, steps, warmup, ext):
    for _ in range(warmup):
        ctx.batch_md_steps(systems, block)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(steps):
        ctx.batch_md_steps(systems, block)
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    return sum(s.n for s in systems) * block * steps / (ms * 1e-3), ms / steps


def run_c1(args, gems, torch, ctx, ext):
    """LJ fluid, 4000 atoms, NVE velocity Verlet: FP64, mixed, and 16 mixed
    replicas; energy drift over the timed steps."""
    from gems_b200 import workloads as W
    w = W.lj_fluid()
    out = {}
    for name, prec, nrep in (("fp64", gems.PREC_FP64, 1), ("mixed", gems.PREC_MIXED, 1),
                             ("batched", gems.PREC_MIXED, 16)):
        ss = []
        for k in range(nrep):
            wk = W.lj_fluid(seed=1 + k)
            g = gems.System(wk["pos"], 1.0, ctx=ctx, vel=wk["vel"])
            g.set_box(wk["L"], (True, True, True))
            e, sg, rc, sh = wk["lj"]
            g.set_lj(e, sg, rc, eshift=sh)
            g.set_skin(wk["skin"])
            g.set_precision(prec)
            g.set_vv(wk["dt"])
            g.interact()
            if k == 0:
                g.tuned = g.autotune(5)
            else:
                g.set_lanes(*ss[0].tuned[:2])
                g.tuned = ss[0].tuned
            ss.append(g)
        e0 = sum(x.energy()[0] + x.energy()[1] for x in ss)
        val, ms = _time_md(ctx, torch, ss, args.block, args.steps, args.warmup, ext)
        e1 = sum(x.energy()[0] + x.energy()[1] for x in ss)
        out[name] = {"value": val, "ms_per_block": ms, "atoms": sum(x.n for x in ss),
                     "drift_ev_per_atom": (e1 - e0) / sum(x.n for x in ss),
                     "lanes_variant": list(ss[0].tuned[:2])}
        for g in ss:
            g.destroy()
    _line("atom-steps/s (LJ fluid 4000, NVE VV)", out["batched"]["value"], UNIT, args,
          {"workload": "lj_fluid_4000 (fcc 10^3, rho*=0.8442, T*=0.72, rc 2.5 shifted, skin 0.3)",
           "md_steps_per_bench_step": args.block}, dtype="f32+f64acc", arms=out,
          **({} if args.no_cpu else {"cpu_baseline": cpu_baseline_c1(args.cpu_seconds)}))


def tersoff_counts(g, L, R_plus_D):
    """Bonds (r <= R+D) and ordered bond pairs (triplets) per system from its
    current list, and the algorithmic counts of one Tersoff evaluation:
      bytes: own position 16 (fixed point) + list 4 n + force 32 + energy 8
             per atom (the force-kernel row of the byte model, float4 reads);
      FP32 flops: per bond ~30 (geometry, cut-off, bond order), per triplet
             ~45 (zeta term, its gradients for i, j and k);
      MUFU: per bond 2 exponentials (FP64 here), per triplet 1 reciprocal."""
    nn, lst = g.neighbour_list()
    x = g.pos
    i = np.repeat(np.arange(g.n), nn)
    j = np.concatenate([lst[:c, a] for a, c in enumerate(nn)]).astype(np.int64)
    d = x[j] - x[i]
    Lv = np.asarray(L, dtype=np.float64)
    d -= Lv * np.round(d / Lv)
    bond = np.sqrt((d * d).sum(1)) <= R_plus_D
    nb = np.bincount(i[bond], minlength=g.n)
    bonds, trip = int(nb.sum()), int((nb * (nb - 1)).sum())
    return {"atoms": g.n, "list_entries": int(nn.sum()), "bonds": bonds, "triplets": trip,
            "bytes": g.n * (16 + 32 + 8) + 4 * int(nn.sum()),
            "flops": 30 * bonds + 45 * trip, "mufu": 2 * bonds + trip}


def run_c5(args, gems, torch, ctx, ext):
    """Tersoff Si(C), 1,000,000 atoms on a diamond lattice, NVE VV dt=1 fs."""
    from gems_b200 import workloads as W
    w = W.tersoff_si()
    out = {}
    want = set(args.arms.split(","))
    for name, prec in (("fp64", gems.PREC_FP64), ("mixed", gems.PREC_MIXED)):
        if name not in want:
            continue
        g = gems.System(w["pos"], w["mass"], ctx=ctx, vel=w["vel"])
        g.set_box(w["L"], (True, True, True))
        g.set_tersoff(w["tersoff"])
        g.set_skin(w["skin"])
        g.set_precision(prec)
        g.set_vv(w["dt"])
        g.interact()
        tuned = g.autotune(5)
        ep0, ek0, _ = g.energy()
        val, ms = _time_md(ctx, torch, [g], args.block, args.steps, args.warmup, ext)
        ep1, ek1, _ = g.energy()
        kern = g.time_kernels(5)
        nsteps = args.block * (args.steps + args.warmup)
        out[name] = {"value": val, "ms_per_block": ms, "atoms": g.n, "steps_run": nsteps,
                     "etot_drift_ev_per_atom": ((ep1 + ek1) - (ep0 + ek0)) / g.n,
                     "bonds_kernel_ms": kern[0], "gather_kernel_ms": kern[1],
                     "force_kernel_ms": kern[0] + kern[1], "rebuild_ms": kern[2], "rebuilds": g.nupd,
                     "lanes_variant": list(tuned[:2])}
        if name == "mixed":
            cts = tersoff_counts(g, w["L"], w["tersoff"][9] + w["tersoff"][10])
            hbm, kind = measured_peaks()
            pk = gems.measure_peaks(torch.cuda.current_device())
            t_ms = kern[0] + kern[1]
            roofs = {"hbm_us": cts["bytes"] / (hbm * 1e9) * 1e6,
                     "fp32_us": cts["flops"] / (pk["fp32_tflops"] * 1e12) * 1e6,
                     "mufu_us": cts["mufu"] / (pk["ex2_gops"] * 1e9) * 1e6}
            bind = max(roofs, key=roofs.get)
            traffic = None
            tpath = os.path.join(ROOT, "profiles", "traffic.json")
            if os.path.exists(tpath):
                with open(tpath) as f:
                    tj = json.load(f)
                if "k_tsf_bonds" in tj and "k_tsf_gather" in tj:
                    traffic = (tj["k_tsf_bonds"]["dram_bytes_per_atom"] +
                               tj["k_tsf_gather"]["dram_bytes_per_atom"]) * g.n
            roof = {"bound": "hbm", "achieved": cts["bytes"] / (t_ms * 1e-3) / 1e9, "peak": hbm,
                    "unit": "GB/s", "frac": cts["bytes"] / (t_ms * 1e-3) / 1e9 / hbm, "traffic": traffic,
                    "peak_source": kind, "kernel": "k_tsf_bonds + k_tsf_gather (one 1M-atom evaluation)",
                    "ms_per_launch": t_ms, "counts": cts, "roof_times_us": roofs, "binding": bind.replace("_us", ""),
                    "frac_of_binding_roof": roofs[bind] / (t_ms * 1e3), "compute_peaks": pk}
        g.destroy()
    head = out["mixed"] if "mixed" in out else out["fp64"]
    extra = {"roofline": roof} if "mixed" in out else {}
    _line("atom-steps/s (Tersoff Si 1M, NVE VV)", head["value"], UNIT, args,
          {"workload": "tersoff_si_1000000 (diamond 50^3, a=5.431, 1000 K, dt 1 fs, skin 1.0)",
           "md_steps_per_bench_step": args.block}, dtype="f32+f64acc", arms=out, **extra,
          **({} if args.no_cpu else {"cpu_baseline": cpu_baseline_c5(args.cpu_seconds)}))


def run_c3(args, gems, torch, ctx, ext):
    """1024 free Au clusters relaxed with FIRE in one batch, then 64
    replica-exchange replicas of a 147-atom cluster (200-900 K).  Under
    torchrun every rank relaxes its own 1024 clusters and holds 64 replicas of
    one ladder of 64 x ranks temperatures; the exchange all-gathers energies."""
    from gems_b200 import workloads as W
    from gems_b200.remd import ReplicaExchange
    rank, world, _ = dist_env()
    tdist = None
    if world > 1:
        import torch.distributed as tdist
    sm, m = W.SMATB["Au"], W.MASS["Au"]
    clusters = W.batched_clusters()
    ss = []
    for k, p in enumerate(clusters):
        g = gems.System(p, m, ctx=ctx)
        g.set_smatb(*sm)
        g.set_precision(gems.PREC_MIXED)
        g.set_lanes(4, 1)
        g.set_fire(0.002, 0.02)
        ss.append(g)
    torch.cuda.synchronize()
    if tdist:
        tdist.barrier()
    t0 = time.perf_counter()
    iters = ctx.batch_fire(ss, 1e-3, 5000)
    torch.cuda.synchronize()
    t_fire = max_over_ranks(time.perf_counter() - t0, tdist, "cuda")
    atom_iters = float(sum(int(i) * g.n for i, g in zip(iters, ss)))
    fmax = [g.fmax() for g in ss[:64]]
    fire = {"systems": len(ss) * world, "atoms": sum(g.n for g in ss) * world, "seconds": t_fire,
            "atom_steps_per_s": world * atom_iters / t_fire, "iters_median": float(np.median(iters)),
            "iters_max": int(max(iters)), "converged": int(sum(int(i) < 5000 for i in iters)) * world,
            "fmax_first64_max": max(fmax)}
    for g in ss:
        g.destroy()
    # replica exchange: this rank's 64 replicas of one ladder over all ranks
    nloc = 64
    nrep = nloc * world
    temps = 200.0 * (900.0 / 200.0) ** (np.arange(nrep) / (nrep - 1))
    base = W.cluster(147, np.random.default_rng(147))
    reps = []
    for k in range(nloc):
        gid = rank * nloc + k
        g = gems.System(base, m, ctx=ctx)
        g.set_smatb(*sm)
        g.set_precision(gems.PREC_MIXED)
        g.set_lanes(4, 1)
        g.set_ermak(0.002, 1.0, temps[gid], seed=500 + gid)
        g.interact()
        reps.append(g)
    rex = ReplicaExchange(ctx, reps, temps, seed=77)
    rounds = 10
    torch.cuda.synchronize()
    if tdist:
        tdist.barrier()
    t0 = time.perf_counter()
    for r in range(1, rounds + 1):
        ctx.batch_md_steps(reps, 500)
        rex.exchange(r)
    torch.cuda.synchronize()
    t_rex = max_over_ranks(time.perf_counter() - t0, tdist, "cuda")
    attempted = 0
    for r in range(1, rounds + 1):
        par = 1 if r % 2 == 0 else -1
        attempted += sum(1 for q in range(nrep) if 0 <= (q + par if q % 2 == 0 else q - par) < nrep
                         and (q + par if q % 2 == 0 else q - par) > q)
    rex_d = {"replicas": nrep, "atoms_each": 147, "rounds": rounds, "steps_per_round": 500,
             "seconds": t_rex, "atom_steps_per_s": nrep * 147 * 500 * rounds / t_rex,
             "accepted": rex.accepted, "attempted": attempted, "ranks": world}
    for g in reps:
        g.destroy()
    if rank != 0:
        return
    _line("atom-steps/s (1024 Au clusters FIRE + 64-replica exchange, batched)", fire["atom_steps_per_s"], UNIT,
          args, {"workload": "1024 Au clusters 13-2000 atoms (log-uniform, seed 3) per GPU, FIRE to 1e-3 eV/A cap "
                             "5000; 64 x 147-atom replicas per GPU on one 200-900 K ladder, swaps every 500 steps"},
          dtype="f32+f64acc", fire=fire, replica_exchange=rex_d, n_gpus=world,
          **({} if args.no_cpu or world > 1 else {"cpu_baseline": cpu_baseline_c3(args.cpu_seconds)}))


def run_c4(args, gems, torch, ctx, ext):
    """Served stream: Poisson 200 req/s of Au/Ag/Pt cluster jobs."""
    from gems_b200 import workloads as W
    srv = gems.Server(ctx, max_jobs=384, max_atoms=600000, lanes=4, variant=1, chunk=50)
    stream = list(W.serve_stream(seconds=args.serve_seconds))
    prepared = []
    for j in stream:
        rng = np.random.default_rng(j["pos_seed"])
        a0 = {"Au": 4.078, "Ag": 4.086, "Pt": 3.924}[j["element"]]
        prepared.append((j, W.cluster(j["n"], rng, a=a0, check=False)))
    lat, done_atoms_steps = [], 0.0
    pending = {}
    k = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while k < len(prepared) or pending:
        now = time.perf_counter() - t0
        while k < len(prepared) and prepared[k][0]["t"] <= now:
            j, pos = prepared[k]
            el = j["element"]
            kind = gems.JOB_FIRE if j["kind"] == "fire" else gems.JOB_MD
            jid = srv.submit(pos, W.MASS[el], W.SMATB[el], kind, 5000 if kind == gems.JOB_FIRE else 2000,
                             dt=0.002, temp=j["temp"], gamma=1.0, fmax=1e-3, seed=j["seed"])
            pending[jid] = (j["t"], j["n"])
            k += 1
        running, queued, fin = srv.step()
        if fin or not running:
            now = time.perf_counter() - t0
            for jid in list(pending):
                r = srv.poll(jid)
                if r["state"] == gems.JOB_DONE:
                    t_arr, n = pending.pop(jid)
                    lat.append(now - t_arr)
                    done_atoms_steps += n * r["iters"]
                    srv.forget(jid)
        if not running and not queued and k < len(prepared):
            time.sleep(max(0.0, prepared[k][0]["t"] - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    srv.close()
    lat = np.array(lat)
    _line("serve latency and throughput (Au/Ag/Pt cluster jobs, Poisson 200 req/s)", float(np.percentile(lat, 50)),
          "s (p50 latency)", args,
          {"workload": "Poisson 200 req/s for %.0f s, Au/Ag/Pt clusters 13-5000 atoms, 70%% FIRE / 30%% 2000-step "
                       "Ermak 300-800 K" % args.serve_seconds}, dtype="f32+f64acc",
          higher_is_better=False, p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
          jobs=len(lat), wall_s=wall, throughput_jobs_per_s=len(lat) / wall,
          throughput_atom_steps_per_s=done_atoms_steps / wall)


def run_next(args, gems, torch, ctx, ext):
    """The rows after the hot path, measured beside their CPU restatement:
    the G-JF constant-pressure piston on the 32k-atom Au bulk (FP64 and
    mixed; one system and a batch of 8), batched L-BFGS of 256 147-atom Au clusters, and
    the NEB deck (30 images of a 72-atom Au slab with a Pt adatom, 20
    iterations)."""
    import sys
    from gems_b200 import workloads as W
    from oracle import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import decks
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    press_atm, pg0, pgv, pmass = 1.0, 1.0, 1.0, 1e-3

    def npt_system(seed, prec):
        w = c2_replica(seed)
        g = gems.System(w["pos"], w["mass"], ctx=ctx)
        g.set_box(w["L"], (True, True, True))
        g.set_smatb(*w["smatb"])
        g.set_skin(w["skin"])
        g.set_precision(prec)
        g.set_lanes(2, 1)
        g.set_lgf(w["dt"], w["temp"], press_atm, pg0, pgv, pmass, seed=seed)
        g.interact()
        return g
    out = {}
    for name, nrep, prec in (("npt_fp64", 1, gems.PREC_FP64), ("npt_fp64_batch8", 8, gems.PREC_FP64),
                             ("npt_mixed", 1, gems.PREC_MIXED), ("npt_mixed_batch8", 8, gems.PREC_MIXED)):
        ss = [npt_system(10 + k, prec) for k in range(nrep)]
        val, ms = _time_md(ctx, torch, ss, args.block, args.steps, args.warmup, ext)
        out[name] = {"value": val, "unit": UNIT, "ms_per_block": ms, "atoms": sum(x.n for x in ss),
                     "box_after": list(ss[0].box_now())}
        for g in ss:
            g.destroy()
    w = c2_replica(10)
    s = O.System(w["pos"], w["mass"])
    s.set_box(w["L"], (True, True, True))
    s.set_smatb(*w["smatb"])
    s.set_skin(w["skin"])
    s.set_lgf(w["dt"], w["temp"], press_atm, pg0, pgv, pmass, O.Rng(123456))
    steps, el = _cpu_steps(s, args.cpu_seconds / 2)
    out["npt_cpu"] = {"value": s.n * steps / el, "unit": UNIT, "cores": cores, "kind": "port",
                      "sample": "%d G-JF steps of the 32000-atom workload" % steps}
    # batched L-BFGS: atom-gradient evaluations per second
    sm = W.smatb_bulk(ncell=2)["smatb"]
    rng = np.random.default_rng(5)
    cl = [W.cluster(147, rng, jitter=0.15) + 200.0 for _ in range(256)]
    mass = W.smatb_bulk(ncell=2)["mass"]
    warm = []
    for _ in range(256):  # warm-up batch of the same size: workspace, maps and kernels loaded
        g = gems.System(W.cluster(147, rng, jitter=0.15) + 200.0, mass, ctx=ctx)
        g.set_smatb(*sm)
        warm.append(g)
    ctx.batch_lbfgs(warm)
    for g in warm:
        g.destroy()
    gs = []
    for p in cl:
        g = gems.System(p, mass, ctx=ctx)
        g.set_smatb(*sm)
        gs.append(g)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stt, its, nfs, _ = ctx.batch_lbfgs(gs)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    nfun = int(np.sum(nfs))
    out["lbfgs_batch256"] = {"value": 147 * nfun / el, "unit": "atom-evaluations/s", "systems": 256,
                             "evaluations": nfun, "iterations_max": int(np.max(its)), "seconds": el,
                             "converged": int(np.sum(stt == 0))}
    for g in gs:
        g.destroy()
    t0 = time.perf_counter()
    nf = 0
    for p in cl[:8]:
        o = O.System(p, mass)
        o.set_smatb(*sm)
        st, it, nfo, em = o.lbfgs()
        nf += nfo
    el = time.perf_counter() - t0
    out["lbfgs_cpu"] = {"value": 147 * nf / el, "unit": "atom-evaluations/s", "cores": cores, "kind": "port",
                        "sample": "L-BFGS of the first 8 clusters"}
    # NEB deck
    d = decks.neb_deck()
    g = gems.System(d["pos"], d["mass"], d["types"], 2, ctx=ctx)
    decks.neb_setup(g, d)
    imgs = decks.neb_fixed_images(g, d, lambda x: x.lbfgs())
    g.destroy()
    images = []
    for k in range(d["nimg"]):
        x = gems.System(imgs[k], d["mass"], d["types"], 2, ctx=ctx)
        decks.neb_setup(x, d)
        images.append(x)
    ctx.neb(images, d["fixed"], d["k"], d["iters"])  # the deck's band (warm-up)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = 10
    for _ in range(reps):  # the band continues from where it is
        ctx.neb(images, d["fixed"], d["k"], d["iters"])
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    out["neb_deck"] = {"value": reps * d["nimg"] * d["iters"] / el, "unit": "image-iterations/s",
                       "seconds": el, "repeats": reps}
    for x in images:
        x.destroy()
    o = O.System(d["pos"], d["mass"], d["types"], 2)
    decks.neb_setup(o, d)
    oi = decks.neb_fixed_images(o, d, lambda x: x.lbfgs())
    t0 = time.perf_counter()
    o.neb(oi, d["fixed"], d["k"], d["iters"])
    el = time.perf_counter() - t0
    out["neb_cpu"] = {"value": d["nimg"] * d["iters"] / el, "unit": "image-iterations/s", "cores": cores,
                      "kind": "port", "sample": "the whole band"}
    _line("atom-steps/s (32000-atom Au bulk under the G-JF piston, FP64)", out["npt_fp64"]["value"], UNIT, args,
          {"workload": "smatb_au_bulk_32000 G-JF NPT (300 K, 1 atm, gamma 1/ps, piston gamma 1/ps, mass 1e-3); "
                       "lbfgs 256 x Au147; neb.gms", "md_steps_per_bench_step": args.block},
          dtype="f64", rows=out, cpu_baseline=out["npt_cpu"])


def main():
    global FIXED_TUNE
    args = parse()
    if args.tune:
        FIXED_TUNE = tuple(int(v) for v in args.tune.split(","))
    if args.impl == "reference":
        run_reference(args)
        return
    if args.config != "c2":
        import torch
        import gems_b200 as gems
        rank, world, local = dist_env()
        if args.config == "c3" and world > 1:
            # replica exchange across ranks: one all-gather of energies per round
            import datetime
            import torch.distributed as tdist
            torch.cuda.set_device(local)
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        elif world > 1:
            if rank == 0:
                print(json.dumps({"config": args.config, "unavailable": "multi-GPU runs cover c2 and c3"}))
            return
        else:
            torch.cuda.set_device(0)
        dev = torch.cuda.current_device()
        ctx = gems.Context(device=dev)
        ext = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
        {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5, "next": run_next}[args.config](
            args, gems, torch, ctx, ext)
        ctx.close()
        if world > 1:
            tdist.barrier()
            tdist.destroy_process_group()
        return
    import torch
    import gems_b200 as gems

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    ctx = gems.Context(device=dev)
    ext = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    blk = args.block
    arms = {}
    want = set(args.arms.split(","))
    if want != {"fp64", "mixed", "batched"}:
        # profiling run: time the requested arms only, print a short line
        w = c2_replica(2)
        out = {}
        for name in ("fp64", "mixed", "batched"):
            if name not in want:
                continue
            prec = gems.PREC_FP64 if name == "fp64" else gems.PREC_MIXED
            nrep = args.replicas if name == "batched" else 1
            first = make_system(gems, ctx, c2_replica(100) if nrep > 1 else w, prec, seed=100)
            ss = [first] + [make_system(gems, ctx, c2_replica(100 + k), prec, seed=100 + k, tune=first.tuned,
                                        therm=0) for k in range(1, nrep)]
            if nrep > 1:
                ctx.batch_md_steps(ss[1:], THERM_STEPS)
            for s_ in ss:
                s_.interact()
            ts, nl = timed_blocks(ctx, torch, ss, blk, args.steps, args.warmup, flush, ext)
            out[name] = {"atom_steps_per_s": sum(x.n for x in ss) * blk * len(ts) / (sum(ts) * 1e-3),
                         "launches": nl}
            for s_ in ss:
                s_.destroy()
        if "rebuild" in want:
            # the list rebuild of the batch on its own (for ncu): replicas of the
            # lattice displaced by N(0, 0.1 A), one list build each, then three
            # forced rebuilds of all of them together
            ss = []
            for k in range(args.replicas):
                wk = c2_replica(100 + k)
                wk["pos"] = np.mod(wk["pos"] + np.random.default_rng(k).normal(0.0, 0.1, wk["pos"].shape),
                                   np.asarray(wk["L"], dtype=np.float64))
                ss.append(make_system(gems, ctx, wk, gems.PREC_MIXED, seed=100 + k, tune=(1, 2), therm=0))
            kb = ctx.batch_time_kernels(ss, 3)
            out["rebuild"] = {"atoms": sum(x.n for x in ss), "rebuild_ms": float(kb[2])}
            for s_ in ss:
                s_.destroy()
        print(json.dumps({"profile_arms": out}), flush=True)
        ctx.close()
        return
    # --- single-system arms
    w = c2_replica(2 + 1000 * rank)
    for name, prec in (("fp64", gems.PREC_FP64), ("mixed", gems.PREC_MIXED)):
        s = make_system(gems, ctx, w, prec, seed=7 + rank)
        s.interact()
        if dist:
            dist.barrier()
        ts, nl = timed_blocks(ctx, torch, [s], blk, args.steps, args.warmup, flush, ext)
        arms[name] = {"value": s.n * blk * len(ts) / (sum(ts) * 1e-3), "ms_per_block": sum(ts) / len(ts),
                      "atoms": s.n, "launches": nl, "lanes_variant": list(s.tuned[:2])}
        if name == "mixed":
            kern = s.time_kernels(50)
            mixed_sys = s
        else:
            kern64 = s.time_kernels(50)
            therm_state = (s.pos, s.vel, s.acel)
            s.destroy()
    # --- batched arm: replicas in one launch
    reps = [make_system(gems, ctx, c2_replica(100 + k + 1000 * rank), gems.PREC_MIXED, seed=100 + k,
                        tune=(2, 0), therm=0) for k in range(args.replicas)]
    ctx.batch_md_steps(reps, THERM_STEPS)  # thermalised together
    if FIXED_TUNE is None:
        ctx.batch_autotune(reps, 10)   # the batch's own best launch shape
    for s in reps:
        s.interact()
    clocks = Clocks(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ts, nl = timed_blocks(ctx, torch, reps, blk, args.steps, args.warmup, flush, ext)
    torch.cuda.synchronize()
    ck = clocks.stop()
    natoms = sum(s.n for s in reps)
    tot_ms = max_over_ranks(sum(ts), dist, "cuda")
    value = world * natoms * blk * len(ts) / (tot_ms * 1e-3)
    arms["batched"] = {"value": natoms * blk * len(ts) / (sum(ts) * 1e-3), "ms_per_block": sum(ts) / len(ts),
                       "atoms": natoms, "replicas": len(reps), "launches": nl,
                       "lanes_variant": list(reps[0].tuned[:2])}
    # --- batched FP64 arm: the same replicas in the plain FP64 kernels, so
    # the headline splits into batching (batched_fp64 / fp64) and precision
    # inside the batch (batched / batched_fp64)
    reps64 = [make_system(gems, ctx, c2_replica(100 + k + 1000 * rank), gems.PREC_FP64, seed=100 + k,
                          tune=(1, 1), therm=0) for k in range(args.replicas)]
    ctx.batch_md_steps(reps64, THERM_STEPS)
    if FIXED_TUNE is None:
        ctx.batch_autotune(reps64, 10)
    for s in reps64:
        s.interact()
    ts64, nl64 = timed_blocks(ctx, torch, reps64, blk, args.steps, args.warmup, flush, ext)
    arms["batched_fp64"] = {"value": natoms * blk * len(ts64) / (sum(ts64) * 1e-3),
                            "ms_per_block": sum(ts64) / len(ts64), "atoms": natoms, "replicas": len(reps64),
                            "launches": nl64, "lanes_variant": list(reps64[0].tuned[:2])}
    for s in reps64:
        s.destroy()
    # --- per-step drop-in e2e (forces on the GPU, integrator on the host)
    dropin = {}
    for name, prec in (("fp64", gems.PREC_FP64), ("mixed", gems.PREC_MIXED)):
        s = make_system(gems, ctx, w, prec, seed=300 + rank, tune=tuple(arms[name]["lanes_variant"]))
        s.interact()
        dropin[name] = timed_dropin(gems, torch, ctx, ext, s, w, max(50, 10 * args.steps))
        s.destroy()
    # --- e2e through the C ABI with host buffers
    te, h2d, d2h = timed_e2e(ctx, torch, reps, blk, args.steps, args.warmup, flush, ext)
    e2e_ms = max_over_ranks(sum(te), dist, "cuda")
    e2e = {"value": world * natoms * blk * len(te) / (e2e_ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    # --- roofline of the dominant kernel: the mixed SMA-TB force pass as the
    # batched arm launches it (all replicas in one launch, its tuned shape)
    nbar = 54.0   # list entries per atom (fcc shells within 6.0 A)
    force_bytes = 16 + 4 + 8 + 4 * nbar + 32 + 8      # own int4, rho^-1/2, rho, list, force, epot
    rho_bytes = 16 + 4 * nbar + 8 + 8 + 4 + 16       # own int4, list, rho, rho^-1/2 (f64, f32), fxe
    peak, peak_kind = measured_peaks()
    kb = ctx.batch_time_kernels(reps, 50)
    ach = force_bytes * natoms / (kb[1] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f)["k_smatb_force_mixed"]["dram_bytes_per_atom"] * natoms
    # compute roofs: measured FP32 / MUFU issue rates against the algorithmic
    # flop and MUFU counts of the same launch
    peaks = gems.measure_peaks(dev)
    sm = c2_replica(2)["smatb"]
    pst = [smatb_pair_stats(r_, c2_replica(2)["L"], sm[5], sm[6]) for r_ in reps]
    tot = {k: sum(p_[k] for p_ in pst) for k in pst[0]}
    c_rho, c_force = smatb_compute_counts(tot)
    roofs = {"peaks": peaks, "pairs_per_launch": tot,
             "force": compute_roof(c_force, force_bytes * natoms, kb[1], peaks, peak),
             "rho": compute_roof(c_rho, rho_bytes * natoms, kb[0], peaks, peak)}
    roofline = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": traffic, "kernel": "k_smatb_force_mixed", "peak_source": peak_kind,
                "bytes_per_launch": force_bytes * natoms, "ms_per_launch": kb[1], "atoms_per_launch": natoms,
                "launch_shape": list(reps[0].tuned[:2]),
                "rho_kernel": {"ms_per_launch": kb[0], "bytes_per_launch": rho_bytes * natoms},
                "rebuild_ms": kb[2], "compute_roofs": roofs,
                "single_32k": {"mixed_force_ms": kern[1], "mixed_rho_ms": kern[0],
                               "fp64_force_ms": kern64[1], "fp64_rho_ms": kern64[0]},
                "note": "working set L2-resident (about 10 MB per replica); the kernel is bound by "
                        "neighbour-gather latency, see profiles/smatb_mixed_batched_8x32k.txt"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / len(ts), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc", "data": "synthetic",
            "config": {"workload": "smatb_au_bulk_32000 x %d replicas (fcc 20^3, a=4.078, Ermak 300 K, "
                                   "gamma 1/ps, dt 2 fs, skin 1.0)" % len(reps),
                       "md_steps_per_bench_step": blk, "replicas_per_gpu": len(reps),
                       "start": "thermalised: %d untimed Ermak steps (4 ps) from the 0 K lattice" % THERM_STEPS,
                       "l2": "flushed between timed blocks (256 MiB write)", "parallelism": "replicas"},
            "arms": arms,
            "speedup_batched_vs_fp64": arms["batched"]["value"] / arms["fp64"]["value"],
            "speedup_mixed_vs_fp64": arms["mixed"]["value"] / arms["fp64"]["value"],
            "speedup_split": {"batching_fp64": arms["batched_fp64"]["value"] / arms["fp64"]["value"],
                              "precision_in_batch": arms["batched"]["value"] / arms["batched_fp64"]["value"],
                              "precision_single": arms["mixed"]["value"] / arms["fp64"]["value"]},
            "e2e": e2e, "e2e_dropin_per_step": dropin,
            "roofline": roofline, "clocks": ck, "gpu_launches": nl}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds, therm_state)
    if rank == 0:
        print(json.dumps(line), flush=True)
    for s in reps:
        s.destroy()
    mixed_sys.destroy()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
