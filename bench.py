#!/usr/bin/env python
"""Throughput of mfa's per-timestep force and integration loop on B200.

Metric: bead-steps/s (beads x time steps / second), mixed precision (FP32 pair
and bond forces, FP64 positions / velocity Verlet / reductions), with the plain
FP64 GPU path reported beside it.

Workload (default): polymer brush with explicit solvent -- 32 x 32 chains of 64
beads end-grafted on a square lattice at 0.3 sigma^-2 (Lx = Ly = 58.42), 9-3
walls at z = 0 and 60 (cutoff 2.5), FENE k = 30 R0 = 1.5, bending k_b = 2,
WCA everywhere, solvent to total density 0.85 (174,080 beads), DPD gamma = 4.5
kT = 1, dt = 0.005, skin and cells autotuned.  Synthetic seeded configuration;
one replica per GPU (weak scaling, no data exchange between ranks).

Timing: W untimed warm-up steps; K timed steps in mfa_step calls of --chunk
steps, each call bracketed by CUDA events on the context's stream, with L2
flushed (a 256 MiB write on the same stream) between calls; barrier +
synchronize around the loop; max over ranks.
`e2e` is the same metric through the public API with host buffers, on the wall
clock: the initial state uploaded from pinned host memory, mfa_step calls of
--chunk steps, each followed by an asynchronous copy of its steps' energies
(the device energy log: step, e_total, v_total, t_fluid of every step) into
pinned host memory, the final state downloaded into pinned host memory, the
scalars and error flags read once.

--impl reference runs the CPU restatement of the reference's loop (serial, one
core, like the Fortran program) on the same workload.
"""
import argparse
import json
import os
import platform
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bead-steps/s"


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--chunk", type=int, default=10, help="time steps per timed iteration (one mfa_step call)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="brush", choices=["brush", "melt", "charged", "batch", "adjoint"])
    ap.add_argument("--n-sys", type=int, default=64, help="systems of the batch workload")
    ap.add_argument("--equil", type=int, default=10000, help="untimed relaxation steps of the fresh configuration")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--drift", action="store_true",
                    help="energy drift of FP64 vs mixed over --drift-steps NVE steps (not a throughput run)")
    ap.add_argument("--drift-steps", type=int, default=100000)
    ap.add_argument("--drift-equil", type=int, default=20000)
    ap.add_argument("--dt", type=float, default=None,
                    help="time step of the --drift runs (default: the configuration's 0.005); the DPD "
                         "noise amplitude follows it (sig = sqrt(2 kT gamma / dt), init_params.f90:845)")
    ap.add_argument("--wall-cut", type=float, default=None,
                    help="9-3 wall cutoff of the brush workload for --drift (default: the configuration's "
                         "2.5; 0: no cutoff, the reference's uncut wall)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the --kernel-times run")
    ap.add_argument("--fixed-skin", type=float, default=None,
                    help="--kernel-times: this skin (and the finest cells for it) after the autotuner, so that "
                         "two builds are compared at equal list lengths")
    ap.add_argument("--energy-every", type=int, default=0,
                    help="--kernel-times: record the energies every this many steps (the device energy log), "
                         "as a driver that reads them would")
    ap.add_argument("--shape", default=None,
                    help="K,BLOCK,SPLIT: after the autotuner, run the pair kernel untiled with this shape (list "
                         "entries per lane and round, threads per block, pieces per chunk), e.g. 2,128,1 -- so "
                         "that a profiled run, whose timings the profiler perturbs, runs the shape an unprofiled "
                         "run picks")
    ap.add_argument("--kernel-times", action="store_true",
                    help="device time of every kernel inside the time-step loop (CUPTI through the torch "
                         "profiler, no serialisation), per step; not a throughput run")
    return ap.parse_args()


def kernel_times(a):
    """Per-kernel device times of the time-step loop as it runs (captured
    graphs, the cooperative rebuild kernel, L2 warm): --steps steps in --chunk-step
    mfa_step calls after the same relaxation and autotuning as the throughput
    run.  The activity records of CUPTI time each kernel without replaying or
    serialising it.  Prints one JSON line."""
    import collections
    import torch
    from torch.profiler import ProfilerActivity, profile
    from mfa_b200 import _abi
    from mfa_b200.api import System
    from mfa_b200.tune import autotune, set_shape
    cfg, meta = make_config(a.workload, a.seed)
    prec = _abi.FP64 if a.precision == "fp64" else _abi.MIXED
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec, device=0)
    if cfg.params.charged:
        g.ewald_k(0)
    g.init_forces()
    if a.equil:
        g.step(a.equil)
    autotune(g)
    if a.shape:
        k, b, sp = (int(x) for x in a.shape.split(","))
        set_shape(g, k, b, False, 0, sp)
    if a.fixed_skin is not None:
        from mfa_b200.tune import cells_for
        g.set_cells(cells_for(g.params, a.fixed_skin), a.fixed_skin)
    if a.energy_every:
        g.set_energy_log(a.energy_every, (a.steps + a.warmup) // a.energy_every + 64)
    for _ in range(max(3, a.warmup // a.chunk)):
        g.step(a.chunk)
    g.sync()
    s0 = g.scalars()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(a.steps // a.chunk):
            g.step(a.chunk)
        g.sync()
        torch.cuda.synchronize()
    s1 = g.scalars()
    steps = (a.steps // a.chunk) * a.chunk
    agg = collections.defaultdict(lambda: [0, 0.0])
    durs = collections.defaultdict(list)
    spans = []
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            agg[ev.name][0] += 1
            agg[ev.name][1] += getattr(ev, "device_time_total", 0.0)
            durs[ev.name].append(ev.time_range.end - ev.time_range.start)
            spans.append((ev.time_range.start, ev.time_range.end, short_name(ev.name)))
    total = sum(t for _, t in agg.values())

    def pct(x, q):
        x = sorted(x)
        return round(x[min(len(x) - 1, int(q * len(x)))], 2)
    rows = [{"kernel": k, "launches": n, "total_us": round(t, 1), "mean_us": round(t / n, 2),
             "us_per_step": round(t / steps, 2), "share": round(t / total, 4),
             "p10_p50_p90_max_us": [pct(durs[k], 0.1), pct(durs[k], 0.5), pct(durs[k], 0.9), pct(durs[k], 1.0)]}
            for k, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1])]
    # idle device time between consecutive kernels of the loop (graph-node
    # and conditional-node latency), by (previous -> next) kernel
    spans.sort()
    gaps = collections.defaultdict(lambda: [0, 0.0])
    for (s0_, e0, n0), (s1_, e1, n1) in zip(spans, spans[1:]):
        gap = s1_ - e0
        if 0.0 <= gap < 200.0:    # a larger gap is the host between mfa_step calls
            gaps[n0 + " -> " + n1][0] += 1
            gaps[n0 + " -> " + n1][1] += gap
    gap_total = sum(t for _, t in gaps.values())
    span_us = (spans[-1][1] - spans[0][0]) if spans else 0.0
    gap_rows = [{"between": k, "count": n, "mean_us": round(t / n, 2), "us_per_step": round(t / steps, 2)}
                for k, (n, t) in sorted(gaps.items(), key=lambda kv: -kv[1][1])]
    print(json.dumps({"workload": meta["workload"], "precision": a.precision, "beads": cfg.n, "steps": steps,
                      "chunk": a.chunk,
                      "skin": g.params.skin, "n_bin": list(g.params.n_bin),
                      "list_rebuilds": s1["n_rebuilds"] - s0["n_rebuilds"],
                      "kernel_us_per_step": round(total / steps, 2),
                      "first_to_last_kernel_us_per_step": round(span_us / steps, 2),
                      "gap_us_per_step": round(gap_total / steps, 2), "kernels": rows, "gaps": gap_rows[:12]}))
    g.close()
    return 0


def loop_kernel_times(g, steps, chunk):
    """Mean device time (us) and launch count of every kernel over `steps`
    steps of the running loop (mfa_step calls of `chunk` steps, L2 warm),
    from CUPTI's activity records through the torch profiler."""
    import collections
    import torch
    from torch.profiler import ProfilerActivity, profile
    g.sync()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(max(1, steps // chunk)):
            g.step(chunk)
        g.sync()
        torch.cuda.synchronize()
    agg = collections.defaultdict(lambda: [0, 0.0])
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            agg[ev.name][0] += 1
            agg[ev.name][1] += getattr(ev, "device_time_total", 0.0)
    return {k: {"launches": n, "mean_us": t / max(n, 1), "total_us": t} for k, (n, t) in agg.items()}


def short_name(k):
    """A kernel's name without return type, namespace and argument list."""
    k = k.replace("void ", "").replace("(anonymous namespace)::", "")
    depth, out = 0, []
    for ch in k:
        if ch == "(" and depth == 0:
            break
        depth += ch == "<"
        depth -= ch == ">"
        out.append(ch)
    return "".join(out)[:60]


def kernel_stat(kt, key):
    """Launch count and mean time of the kernels whose name contains `key`."""
    n = sum(v["launches"] for k, v in kt.items() if key in k)
    t = sum(v["total_us"] for k, v in kt.items() if key in k)
    return n, (t / n if n else None)


def accuracy_vs_fp64(cfg, st, dev, steps=2000, every=100):
    """The mixed path's reported quantities against the plain FP64 path.

    At one state (the mixed run's last): the force on every bead (max-norm
    relative error), each energy term, and the pair pressure (2 KE + W)/(3 V)
    with W the pair virial sum r_ij . f_ij.  Along a run of `steps` steps from
    that state in both precisions (the same Philox noise, so the two stay
    correlated until chaos separates them): the mean squared radius of
    gyration of the grafted chains and the brush height (mean z of the chain
    beads), sampled every `every` steps, with the difference of the two means
    and the standard error of the FP64 mean (block averages)."""
    import numpy as np
    from mfa_b200 import _abi
    from mfa_b200.api import System
    p = cfg.params
    V = p.boundary[0] * p.boundary[1] * p.boundary[2]
    chain = np.arange(cfg.n) < p.n_chain * p.n_mon
    out, traj = {}, {}
    for name, prec in (("fp64", _abi.FP64), ("mixed", _abi.MIXED)):
        g = System(p, st["r0"], st["v"], cfg.a_type, cfg.mass, q=cfg.q, a=st["a"], mic=st["mic"],
                   precision=prec, device=dev)
        g.init_forces(full=True)
        f = g.download(_abi.F)["force"]
        sc = g.scalars()
        out[name] = {"force": f, "scalars": sc,
                     "pressure": (2.0 * sc["t_fluid"] + sc["virial"]) / (3.0 * V)}
        rg, hz = [], []
        for _ in range(steps // every):
            g.step(every)
            rg.append(float(np.sum(g.observe()["r_g2_brush"])))
            hz.append(float(g.download(_abi.R0)["r0"][chain, 2].mean()))
        traj[name] = (np.array(rg), np.array(hz))
        g.close()
    f64, f32 = out["fp64"]["force"], out["mixed"]["force"]
    s64, s32 = out["fp64"]["scalars"], out["mixed"]["scalars"]
    res = {"force_max_rel": float(np.abs(f32 - f64).max() / np.abs(f64).max())}
    for k in ("v_fluid_fluid", "v_fluid_wall", "v_intra_molec", "v_bend", "v_coul", "v_total"):
        if s64[k] != 0.0:
            res[k + "_rel"] = abs(s32[k] - s64[k]) / abs(s64[k])
    res["pressure_pair"] = out["fp64"]["pressure"]
    res["pressure_pair_rel"] = abs(out["mixed"]["pressure"] - out["fp64"]["pressure"]) / abs(out["fp64"]["pressure"])

    def mean_sem(x):
        b = x[: (len(x) // 5) * 5].reshape(5, -1).mean(axis=1)
        return float(x.mean()), float(b.std(ddof=1) / np.sqrt(5))

    for key, k in (("rg2", 0), ("brush_height_mean_z", 1)):
        m64, e64 = mean_sem(traj["fp64"][k])
        m32, _ = mean_sem(traj["mixed"][k])
        res[key] = {"fp64": m64, "mixed": m32, "diff": m32 - m64, "sem_fp64": e64}
    res["note"] = (f"forces, energies and pressure at one state; rg2 (sum of the per-axis mean square radii "
                   f"of gyration of the grafted chains) and brush height averaged over {steps} steps from it, "
                   f"every {every}")
    return res


def drift(a):
    """Equilibrate with the thermostat (FP64), then run the same state without
    thermostat (NVE) in FP64 and in mixed precision and report the energy
    drift per bead, a linear-fit slope per 1e5 steps and the step time."""
    import numpy as np
    import torch
    from mfa_b200 import _abi
    from mfa_b200.api import System
    import math
    cfg, meta = make_config(a.workload, a.seed, wall_cut=a.wall_cut)
    if a.dt is not None:
        cfg.params.dt = a.dt
        cfg.params.sig = math.sqrt(2.0 * cfg.params.temp * cfg.params.friction / a.dt)
    g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=_abi.FP64)
    g.init_forces()
    g.step(a.drift_equil)
    st = g.download()
    g.close()
    p = cfg.params.copy()
    p.thermostat = _abi.THERMO_NONE
    every = max(1, a.drift_steps // 1000)
    res = {}
    for name, prec in (("fp64", _abi.FP64), ("mixed", _abi.MIXED)):
        h = System(p, st["r0"], st["v"], cfg.a_type, cfg.mass, q=cfg.q, mic=st["mic"], precision=prec)
        h.init_forces(full=True)
        h.set_energy_log(every, a.drift_steps // every + 8)
        ext = torch.cuda.ExternalStream(h.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        h.step(a.drift_steps)
        e1.record(ext)
        h.sync()
        log = h.energy_log()
        t, E, T = log[:, 0], log[:, 1], log[:, 3]
        slope = float(np.polyfit(t, E, 1)[0])
        res[name] = {"drift_per_bead": float((E[-1] - E[0]) / cfg.n),
                     "fit_slope_per_bead_per_1e5_steps": slope * 1e5 / cfg.n,
                     "fluct_rms_per_bead": float(np.std(E) / cfg.n),
                     "kT_mean": float(2.0 * T.mean() / (3.0 * cfg.n)),
                     "ms_per_step": e0.elapsed_time(e1) / a.drift_steps,
                     "bead_steps_per_s": cfg.n * a.drift_steps / (e0.elapsed_time(e1) * 1e-3)}
        h.close()
        # e_total is the reference's sum (verlet_velocities.f90:187): it leaves
        # out the bending and Coulomb energies, so with bending it is not a
        # constant of the motion.  The same run again, read every `every`
        # steps, with those terms added back.
        h = System(p, st["r0"], st["v"], cfg.a_type, cfg.mass, q=cfg.q, mic=st["mic"], precision=prec)
        h.init_forces(full=True)
        ts, Ec = [], []
        for _ in range(a.drift_steps // every):
            h.step(every)
            sc = h.scalars()
            ts.append(sc["i_time"])
            Ec.append(sc["e_total"] + sc["v_bend"] + (sc["v_coul"] if p.charged else 0.0))
        h.close()
        ts, Ec = np.asarray(ts, dtype=np.float64), np.asarray(Ec)
        res[name]["conserved"] = {
            "energy": "e_total + v_bend" + (" + v_coul" if p.charged else ""),
            "drift_per_bead": float((Ec[-1] - Ec[0]) / cfg.n),
            "fit_slope_per_bead_per_1e5_steps": float(np.polyfit(ts, Ec, 1)[0]) * 1e5 / cfg.n,
            "fluct_rms_per_bead": float(np.std(Ec) / cfg.n)}
    print(json.dumps({"mode": "drift", "workload": meta["workload"], "beads": cfg.n, "nve_steps": a.drift_steps,
                      "wall_cut": cfg.params.wall_cut if cfg.params.symmetry == 0 else None,
                      "dt": cfg.params.dt, "equilibration_steps_dpd": a.drift_equil, **res,
                      "mixed_over_fp64_speed": res["mixed"]["bead_steps_per_s"] / res["fp64"]["bead_steps_per_s"]}))
    return 0


def make_config(name, seed, wall_cut=None):
    from mfa_b200 import configs
    if name == "brush":
        kw = {} if wall_cut is None else {"wall_cut": wall_cut}
        return configs.brush(seed=seed, **kw), {
            "workload": "brush_explicit_solvent_32x32x64", "chains": "32x32", "n_mon": 64,
            "grafting_density": 0.3, "wall_gap": 60.0, "solvent_density": 0.85}
    if name == "melt":
        return configs.melt(seed=seed), {"workload": "melt_100x32", "chains": 100, "n_mon": 32}
    return configs.charged(seed=seed), {"workload": "polyelectrolyte_200x50_ewald", "chains": 200,
                                         "n_mon": 50, "n_kmax": 10}


def cpu_info():
    model = platform.processor()
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count()


def run_oracle(cfg, seconds, max_steps, warm=2):
    """The CPU restatement (serial, like the reference) on the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle
    o = Oracle(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, list_cap=512, rng_mode=1)
    o.init_forces()
    for _ in range(warm):
        o.md_step()
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and (time.perf_counter() - t0) < seconds:
        o.md_step()
        steps += 1
    dt = time.perf_counter() - t0
    return cfg.n * steps / dt, steps, dt


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the loop runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.window = (0.0, float("inf"))

    def mark(self, begin, end):
        """Only samples taken between these host times describe the timed region."""
        self.window = (begin, end)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def wait_first(self, limit_s):
        """Block until nvidia-smi has printed its first sample (or limit_s
        passed), so that the sampler is running when the timed region opens."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < limit_s:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        b, e = self.window
        inside = [ln for ts, ln in self.lines if b <= ts <= e + 0.2]
        where = "inside the timed region"
        if not inside and self.lines:
            # a timed region shorter than the sampling period (100 ms): the
            # samples nearest to it, one on each side where there are two
            before = [ln for ts, ln in self.lines if ts < b]
            after = [ln for ts, ln in self.lines if ts > e]
            inside = before[-1:] + after[:1]
            where = (f"timed region of {1e3 * (e - b):.1f} ms is shorter than the 100 ms sampling "
                     "period: the nearest sample on each side of it")
        for ln in inside:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, flag in zip(names, parts[4:8]):
                if flag.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "where": where if sm else "no sample arrived"}


def pair_work(g, cfg):
    """Counts behind the algorithmic figures of one pair-kernel launch: listed
    half-pairs, in-cutoff half-pairs and the sum of list rows (binning's half
    list holds every pair once)."""
    import numpy as np
    from mfa_b200 import _abi
    p = cfg.params
    st = g.download(_abi.R0)
    cell, cnt, nbr = g.debug_lists(int(g.scalars()["max_neigh"]) + 1)
    r = st["r0"]
    t = cfg.a_type
    ii = np.repeat(np.arange(cfg.n), cnt)
    jj = nbr[np.arange(nbr.shape[1])[None, :] < cnt[:, None]] - 1
    d = r[ii] - r[jj]
    for k in range(3):
        if k < 2 or p.symmetry == 1:
            L = p.boundary[k]
            d[:, k] -= L * np.trunc(2.0 * d[:, k] / L)
    r2 = (d * d).sum(1)
    rc2 = np.array(p.range_2[:]).reshape(8, 8)[t[ii] - 1, t[jj] - 1]
    inside = int((r2 < rc2).sum())
    out = {"listed_half_pairs": int(cnt.sum()), "incut_half_pairs": inside, "list_entries": int(cnt.sum())}
    if p.charged:
        # Ewald real space: inside the LJ range (reference form) or to its own cutoff
        out["ewald_real_pairs"] = inside if (p.quirks & _abi.Q_EWALD_REAL_IN_LJ) else int((r2 < p.ewald_rc_2).sum())
    return out


def batch_bench(a):
    """Uneven implicit-solvent brushes (default 64 systems, ~0.95 M beads)
    advanced together (mfa_batch_step): each kernel stage of a step is one
    grouped launch for all systems, captured graphs (with MFA_BATCH_PERSIST=1:
    each call of --chunk steps is one persistent cooperative launch).  Beside it: the
    same systems stepped one after another through mfa_step (one system per
    launch sequence), FP64, and the serial CPU restatement on a sample of the
    systems."""
    import numpy as np
    import torch
    from mfa_b200 import _abi, configs
    from mfa_b200.api import Batch, System
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = local
    torch.cuda.set_device(dev)
    # whole systems are the unit of work, shared out by bead count (greedy,
    # largest first to the least-loaded rank; the same partition on every rank)
    from mfa_b200.ranks import max_over_ranks, shard_by_weight, sum_over_ranks
    every_sys = configs.uneven_brushes(seed=a.seed, n_sys=a.n_sys)
    my_ids = shard_by_weight(list(range(len(every_sys))), [c.n for c in every_sys], rank, world)
    cfgs = [every_sys[k] for k in my_ids]
    n = sum(c.n for c in cfgs)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")

    def make(prec):
        ss = []
        for c in cfgs:
            g = System(c.params, c.r0, c.v, c.a_type, c.mass, precision=prec, device=dev)
            g.init_forces()
            ss.append(g)
        return ss

    def timed_batch(prec, steps, warmup):
        ss = make(prec)
        b = Batch(ss)
        if a.equil:
            b.step(a.equil)
        ext = torch.cuda.ExternalStream(b.stream_ptr(), device=f"cuda:{dev}")
        sampler = ClockSampler(dev)
        sampler.start()
        chunks = [a.chunk] * (steps // a.chunk) + ([steps % a.chunk] if steps % a.chunk else [])
        # at least three warm-up calls of each timed call length (graphs captured before timing)
        warm_calls = [a.chunk] * max(3, -(-warmup // a.chunk))
        warm_calls += [ln for ln in sorted(set(chunks)) if ln != a.chunk for _ in range(3)]
        for k, ln in enumerate(warm_calls):
            with torch.cuda.stream(ext):
                flush.fill_(k & 0xff)
            b.step(ln)
        b.sync()
        sampler.wait_first(5.0)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in chunks]
        l0 = b.launches()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t_begin = time.time()
        for k, nst in enumerate(chunks):
            with torch.cuda.stream(ext):
                flush.fill_(k & 0xff)
            ev[k][0].record(ext)
            b.step(nst)
            ev[k][1].record(ext)
        b.sync()
        torch.cuda.synchronize(dev)
        sampler.mark(t_begin, time.time())
        clocks = sampler.stop()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
        launches = b.launches() - l0
        timed_batch.calls = len(chunks)
        sc = b.scalars()
        errs = sum(1 for x in sc if x["error_bits"])
        b.close()
        for g in ss:
            g.close()
        return ms, launches, clocks, errs, sc

    ms_mixed, launches, clocks, errs, sc_mixed = timed_batch(_abi.MIXED, a.steps, a.warmup)
    # the per-system scalars of every rank in one table (one collective)
    from mfa_b200.ranks import gather_system_values
    table = gather_system_values([[x["e_total"], x["t_fluid"], float(x["error_bits"] != 0)] for x in sc_mixed],
                                 my_ids, len(every_sys), dist, f"cuda:{dev}")
    ms_max = max_over_ranks(ms_mixed, dist, f"cuda:{dev}")
    n_all = int(sum_over_ranks(n, dist, f"cuda:{dev}"))
    value = n_all * a.steps / (ms_max * 1e-3)
    ms_fp64, _, _, _, _ = timed_batch(_abi.FP64, a.steps, a.warmup)
    ms_fp64 = max_over_ranks(ms_fp64, dist, f"cuda:{dev}")
    # the same systems one after another (a launch sequence per system)
    ss = make(_abi.MIXED)
    st = torch.cuda.Stream(device=f"cuda:{dev}")
    for g in ss:
        g.step(a.chunk)
    torch.cuda.synchronize(dev)
    seq_steps = max(a.chunk, a.steps // 4)
    t0 = time.perf_counter()
    for g in ss:
        g.step(seq_steps)
    for g in ss:
        g.sync()
    t_seq = time.perf_counter() - t0
    for g in ss:
        g.close()
    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu:
            # serial CPU restatement on a sample: the smallest systems, a few steps each
            import statistics
            sample = sorted(cfgs, key=lambda c: c.n)[:8]
            tot, done = 0.0, 0
            for c in sample:
                rate, steps, dt = run_oracle(c, a.cpu_seconds / len(sample), 1000)
                tot += dt
                done += c.n * steps
            model, ncpu = cpu_info()
            cpu = {"value": done / tot, "unit": METRIC, "cores": 1, "kind": "port",
                   "sample": f"{len(sample)} smallest systems of the batch, serial C restatement of the "
                             f"reference loop one system after another, 1 core of {model} ({ncpu} host threads)"}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator, no reference data)",
            "config": {"workload": f"uneven_implicit_brushes_x{a.n_sys}", "systems_per_gpu": len(cfgs),
                       "beads_per_gpu": n, "beads_total": n_all,
                       "chain_lengths": sorted({c.params.n_mon for c in cfgs}),
                       "grafting_density": [round(min(c.params.n_chain / (c.params.boundary[0] * c.params.boundary[1])
                                                      for c in cfgs), 3),
                                            round(max(c.params.n_chain / (c.params.boundary[0] * c.params.boundary[1])
                                                      for c in cfgs), 3)],
                       "precision": "mixed", "dt": 0.005, "thermostat": "dpd",
                       "steps_per_timed_iteration": a.chunk,
                       "l2": "flushed between timed iterations (256 MiB write); state is larger than L2",
                       "parallelism": f"whole systems over {world} GPU(s) by bead count, no data exchange"},
            "fp64": {"value": n_all * a.steps / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64 / a.steps},
            "mixed_over_fp64": ms_fp64 / ms_max,
            "one_system_at_a_time": {"value": n * seq_steps / t_seq,
                                     "note": "the same systems through mfa_step one after another (wall clock)"},
            "gpu_launches": int(launches),
            "launches_per_call": launches / timed_batch.calls,
            "systems_with_errors": errs,
            "gathered": {"systems": int(table.shape[0]), "systems_with_errors": int(table[:, 2].sum()),
                         "kinetic_temperature_mean": float((2.0 * table[:, 1] / (3.0 * np.array(
                             [c.n for c in every_sys]))).mean()),
                         "note": "per-system e_total, t_fluid and error flag of every rank, one all-reduce"},
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def adjoint_bench(a):
    """Trajectory sensitivities: an implicit-solvent brush of 16 x 16 chains of 64
    beads (16,384 beads, grafting density 0.3, 9-3 walls 60 apart, WCA + FENE,
    DPD gamma = 4.5), 200 steps, checkpoints every 20.  Times, on the context's
    stream: the adjoint (forward with checkpoints, recomputation, backward),
    the same 200 steps forward with the observable (the path the adjoint
    differentiates), and 200 fast-path steps (mfa_step); checks the FP64
    gradient against central differences (h = 1e-4 relative, common random
    numbers)."""
    import math
    import torch
    from mfa_b200 import _abi, configs
    from mfa_b200.api import System
    from mfa_b200.sensitivity import NAMES, base_values, perturbed
    # the brush of the throughput workload (bending k_b = 2 included), 16 x 16 chains, implicit solvent
    cfg = configs.brush(seed=a.seed, nx=16, ny=16, n_mon=64, graft=0.3, z_wall=60.0, solvent=False, k_bend=2.0)
    S, K = 200, 20
    g0 = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, precision=_abi.FP64)
    g0.init_forces(full=True)
    g0.step(a.equil)
    st = g0.download()
    g0.close()

    def fresh(params, prec):
        g = System(params, st["r0"], st["v"], cfg.a_type, cfg.mass, a=st["a"], mic=st["mic"], precision=prec)
        g.binning()
        return g

    def timed(prec, fn, warm=False, reps=3):
        """best of reps (event time on the context's stream) and that run's result"""
        best_ms, best_out = None, None
        for _ in range(reps):
            g = fresh(cfg.params, prec)
            if warm:
                fn(g)        # captures the fast path's graphs outside the timed region
            g.sync()
            ext = torch.cuda.ExternalStream(g.stream_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(ext)
            out = fn(g)
            e1.record(ext)
            g.sync()
            ms = e0.elapsed_time(e1)
            g.close()
            if best_ms is None or ms < best_ms:
                best_ms, best_out = ms, out
        return best_ms, best_out

    res = {}
    for name, prec in (("fp64", _abi.FP64), ("mixed", _abi.MIXED)):
        # first call on a context (allocates its workspace, captures its sequences)
        t_adj, (J, grad) = timed(prec, lambda g: g.adjoint(S, K))
        # a repeated call of the same length (cached workspace and sequences), as
        # the fast path is timed after its graphs are captured
        t_adj_warm, _ = timed(prec, lambda g: g.adjoint(S, K), warm=True)
        t_obs, _ = timed(prec, lambda g: g.trajectory_observable(S))
        t_fast, _ = timed(prec, lambda g: g.step(S), warm=True)
        res[name] = {"J": J, "grad": grad, "adjoint_ms": t_adj, "adjoint_ms_repeated_call": t_adj_warm,
                     "forward_observable_ms": t_obs, "forward_fast_path_ms": t_fast,
                     "adjoint_over_forward": t_adj / t_obs, "adjoint_over_fast_path": t_adj / t_fast,
                     "repeated_adjoint_over_fast_path": t_adj_warm / t_fast}
    # where the mixed adjoint's device time goes: CUPTI activity records of one
    # more adjoint call (after the timed ones: its graphs are captured)
    import collections
    from torch.profiler import ProfilerActivity, profile
    g = fresh(cfg.params, _abi.MIXED)
    g.adjoint(S, K)
    g.sync()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        g.adjoint(S, K)
        g.sync()
        torch.cuda.synchronize()
    g.close()
    agg = collections.defaultdict(lambda: [0, 0.0])
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            agg[short_name(ev.name)][0] += 1
            agg[short_name(ev.name)][1] += getattr(ev, "device_time_total", 0.0)
    adj_total = sum(t for _, t in agg.values())
    adj_kernels = {"kernel_ms": round(adj_total / 1e3, 3),
                   "top": [{"kernel": k, "launches": n, "ms": round(t / 1e3, 3), "share": round(t / adj_total, 4)}
                           for k, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1])[:10]]}
    # central differences (FP64) for every parameter
    base = base_values(cfg.params)
    h = 1e-4
    fd = {}
    for nm in NAMES:
        js = []
        for f in (1 + h, 1 - h):
            g = fresh(perturbed(cfg.params, nm, f), _abi.FP64)
            js.append(g.trajectory_observable(S))
            g.close()
        fd[nm] = (js[0] - js[1]) / (2 * h * base[nm])
    # step-size study for sigma: central differences against h (truncation
    # error falls as h^2, rounding and the chaos of a 200-step trajectory grow
    # as h falls), the adjoint beside them
    fd_sigma = {}
    for hh in (1e-3, 3e-4, 1e-4, 3e-5, 1e-5, 1e-6):
        js = []
        for f in (1 + hh, 1 - hh):
            g = fresh(perturbed(cfg.params, "sigma", f), _abi.FP64)
            js.append(g.trajectory_observable(S))
            g.close()
        fd_sigma[f"{hh:g}"] = (js[0] - js[1]) / (2 * hh * base["sigma"])
    g64 = res["fp64"]["grad"]
    rel = {nm: abs(g64[nm] - fd[nm]) / max(abs(fd[nm]), 1e-30) for nm in NAMES}
    rel32 = {nm: abs(res["mixed"]["grad"][nm] - g64[nm]) / max(abs(g64[nm]), 1e-30) for nm in NAMES}
    print(json.dumps({
        "mode": "adjoint", "metric": "adjoint cost / forward cost (repeated call / fast path)",
        "value": res["mixed"]["repeated_adjoint_over_fast_path"],
        "unit": "ratio", "higher_is_better": False,
        "config": {"workload": "brush_implicit_16x16x64", "beads": cfg.n, "steps": S, "checkpoint_every": K,
                   "k_bend": cfg.params.k_bend,
                   "observable": "time average of <z> + <R_ee^2>", "dt": cfg.params.dt},
        "fp64": res["fp64"], "mixed": res["mixed"], "central_differences_fp64": fd,
        "rel_err_fp64_adjoint_vs_fd": rel, "rel_err_mixed_vs_fp64_adjoint": rel32,
        "fd_step_study_sigma": {"adjoint_fp64": g64["sigma"], "central_differences": fd_sigma},
        "mixed_adjoint_kernels": adj_kernels}))
    return 0


def main():
    a = args_()
    if a.drift:
        return drift(a)
    if a.kernel_times:
        return kernel_times(a)
    if a.workload == "adjoint" and a.impl != "reference":
        return adjoint_bench(a)
    if a.workload == "batch" and a.impl != "reference":
        return batch_bench(a)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return 0
        if a.workload == "batch":
            print(json.dumps({"impl": "reference", "unavailable": "the batch workload has no single reference "
                              "run; its CPU baseline is the serial restatement per system (cpu_baseline)"}))
            return 0
        cfg, meta = make_config(a.workload, a.seed)
        # each step is one full time step of the workload; the run is capped at
        # about two minutes of CPU time (the step count reported is what ran)
        rate, steps, dt = run_oracle(cfg, seconds=120.0, max_steps=a.steps, warm=min(a.warmup, 3))
        model, ncpu = cpu_info()
        line = {
            "impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": a.gpus,
            "steps": steps, "warmup": a.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(meta, beads=cfg.n, dt=cfg.params.dt, skin=cfg.params.skin),
            "cpu_baseline": {"value": rate, "unit": METRIC, "cores": 1, "kind": "port",
                             "sample": f"{steps} full time steps of the {cfg.n}-bead workload, serial C restatement "
                                       f"of the Fortran loop on 1 core ({model}, {ncpu} host threads)"},
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch
    from mfa_b200 import _abi
    from mfa_b200.api import System
    from mfa_b200.tune import autotune, set_shape

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = local
    torch.cuda.set_device(dev)
    cfg, meta = make_config(a.workload, a.seed + rank)
    n = cfg.n
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")

    def timed_run(prec, steps, warmup, flush_l2=True):
        g = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=prec, device=dev)
        if cfg.params.charged:
            g.ewald_k(0)
        g.init_forces()
        if a.equil:
            g.step(a.equil)
        tuned = autotune(g)
        shapes = tuned["pair_shape"]
        g.tuned = min(shapes, key=shapes.get)
        if a.shape:
            k, b, sp = (int(x) for x in a.shape.split(","))
            set_shape(g, k, b, False, 0, sp)
            g.tuned = (k, b, False, 0, sp)
        g.tuning = {f"{k}x{b}{'-tiled' if t else ''}{f'-queue{q}' if q else ''}{f'-split{p}' if p > 1 else ''}":
                    round(1e3 * s / 300, 4) for (k, b, t, q, p), s in shapes.items()}
        g.skin_tuning = {f"{s:g}": round(1e3 * v / 300, 4) for s, v in tuned["skin_for_shape"].items()}
        g.skin_tuning_first = {f"{s:g}": round(1e3 * v / 300, 4) for s, v in tuned["skin"].items()}
        ext = torch.cuda.ExternalStream(g.stream_ptr(), device=f"cuda:{dev}")
        # a timed iteration is `chunk` consecutive time steps (one mfa_step call:
        # fused velocity/position kernels, captured graphs); L2 is flushed
        # between iterations
        chunks = [a.chunk] * (steps // a.chunk) + ([steps % a.chunk] if steps % a.chunk else [])
        # the clock sampler starts before the warm-up, so that starting
        # nvidia-smi does not overlap the timed region
        sampler = ClockSampler(dev)
        sampler.start()
        # warm-up: W steps rounded up to whole calls, and at least three calls
        # of every length the timed loop uses.  mfa_step captures the graph of
        # a whole call the second time it sees a step count, so three calls
        # put the capture and instantiation before the first timed event.
        lengths = sorted(set(chunks))
        warm_calls = [a.chunk] * max(3, -(-warmup // a.chunk))
        for ln in lengths:
            if ln != a.chunk:
                warm_calls += [ln] * 3
        warm_calls.append(chunks[0])
        for k, ln in enumerate(warm_calls):
            with torch.cuda.stream(ext):
                flush.fill_(k & 0xff)
            g.step(ln)
        g.sync()
        sampler.wait_first(5.0)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in chunks]
        s0 = g.scalars()
        launches0 = s0["kernel_launches"]
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t_begin = time.time()
        torch.cuda.nvtx.range_push(f"timed_{'mixed' if prec == _abi.MIXED else 'fp64'}")
        for k, nst in enumerate(chunks):
            if flush_l2:
                with torch.cuda.stream(ext):
                    flush.fill_(k & 0xff)
            ev[k][0].record(ext)
            g.step(nst)
            ev[k][1].record(ext)
        torch.cuda.nvtx.range_pop()
        g.sync()
        torch.cuda.synchronize(dev)
        sampler.mark(t_begin, time.time())
        clocks = sampler.stop()
        if dist is not None:
            dist.barrier()
        per_call = [e0.elapsed_time(e1) for e0, e1 in ev]
        ms = sum(per_call)
        s = g.scalars()
        s["rebuilds_timed"] = s["n_rebuilds"] - s0["n_rebuilds"]
        srt = sorted(per_call)
        s["per_call_ms"] = {"calls": len(per_call), "steps_per_call": a.chunk,
                            "min": srt[0], "median": srt[len(srt) // 2], "max": srt[-1],
                            "first": per_call[:8]}
        return g, ms, s["kernel_launches"] - launches0, clocks, s

    # headline: mixed precision
    g, ms_mixed, launches, clocks, s_mixed = timed_run(_abi.MIXED, a.steps, a.warmup)
    shape_mixed = g.tuned
    tuning_mixed = g.tuning
    skin_mixed, nbin_mixed, skin_tuning = g.params.skin, list(g.params.n_bin), g.skin_tuning
    from mfa_b200.ranks import max_over_ranks
    ms_max = max_over_ranks(ms_mixed, dist, f"cuda:{dev}")
    value = world * n * a.steps / (ms_max * 1e-3)

    # steady state without flushes: captured 10-step graphs, L2-resident state
    g.sync()
    ext = torch.cuda.ExternalStream(g.stream_ptr(), device=f"cuda:{dev}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    g.step(a.steps)
    e1.record(ext)
    g.sync()
    ms_resident = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{dev}")

    # device time of each kernel inside the running loop (CUPTI activity
    # records: graph nodes as they run, nothing serialised or replayed)
    loop_kt = loop_kernel_times(g, 200, a.chunk)

    # dominant kernel: the pair kernel, timed alone on the context's stream
    work = pair_work(g, cfg)
    # L2 flushed before every `chunk`-th launch, as the timed loop flushes it
    # before every call of `chunk` steps (the launch-average of that loop);
    # and, for reference, flushed before every launch (cold)
    # A spin of ~0.5 ms on the stream after each flush lets the host enqueue
    # the launches that follow before the device reaches them, so the events
    # time the device work and not the host's enqueue rate.
    reps = 2 * a.chunk
    pk, pk_cold = [], []
    torch.cuda.nvtx.range_push("pair_alone")
    for k in range(reps + 5):
        cold = k >= reps
        if cold or k % a.chunk == 0:
            with torch.cuda.stream(ext):
                flush.fill_(k & 0xff)
                torch.cuda._sleep(1_000_000)
        g.zero_forces()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(ext)
        g.pair_forces()      # the time step's pair kernel (9-3 walls fused), adding to force
        p1.record(ext)
        (pk_cold if cold else pk).append((p0, p1))
    torch.cuda.nvtx.range_pop()
    g.sync()
    torch.cuda.synchronize(dev)
    pair_ms = sum(x.elapsed_time(y) for x, y in pk) / len(pk)
    pair_ms_cold = sum(x.elapsed_time(y) for x, y in pk_cold) / len(pk_cold)
    # the neighbour-list rebuild (binning: counting sort + list build), forced
    # through the subroutine entry point, L2 flushed before each
    rb = []
    torch.cuda.nvtx.range_push("rebuild_alone")
    for k in range(5):
        with torch.cuda.stream(ext):
            flush.fill_(k & 0xff)
            torch.cuda._sleep(1_000_000)
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(ext)
        g.binning()
        b1.record(ext)
        rb.append((b0, b1))
    torch.cuda.nvtx.range_pop()
    g.sync()
    rebuild_ms = sum(x.elapsed_time(y) for x, y in rb) / len(rb)
    # algorithmic HBM bytes of one launch: each particle's sorted position and
    # velocity records (16 + 16 B), its row length (4 B), its force record
    # read and written once by the reductions (16 + 16 B) and its list row
    # (4 B per entry)
    pair_bytes = n * (16 + 16 + 4 + 16 + 16) + 4 * work["list_entries"]
    # algorithmic flops (canonical counts): 17 per listed half-pair, 38 (LJ) + 29 (DPD) per in-cutoff half-pair
    # canonical counts: 17 per listed half-pair; LJ 38 per in-cutoff pair; DPD
    # 29 more with that thermostat; Ewald real 20 + erfc + exp (2 each) = 24
    therm = cfg.params.thermostat
    pair_flops = (17 * work["listed_half_pairs"] + (38 + (29 if therm == _abi.THERMO_DPD else 0)) *
                  work["incut_half_pairs"] + 24 * work.get("ewald_real_pairs", 0))
    pair_label = "k_pair (fluid_fluid" + (" + dpd_forces" if therm == _abi.THERMO_DPD else "") + \
                 (" + lgv_forces" if therm == _abi.THERMO_LGV else "") + \
                 (" + ewald_real" if cfg.params.charged else "") + \
                 (" + 9-3 walls" if cfg.params.symmetry == 0 and cfg.params.wall == 2 else "") + ")"
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = pair_bytes / (pair_ms * 1e-3) / 1e9
    traffic, traffic_src = None, None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "pair_traffic.json")))
        if prof.get("workload") == meta["workload"]:
            traffic = prof.get("dram_bytes_per_launch")
            traffic_src = ("stored ncu capture of the same kernel and workload (profiles/pair_traffic.json: "
                           f"{prof.get('command', 'see file')}), not measured in this run")
    except (OSError, ValueError):
        pass
    # integration: the fused velocity-Verlet kernel of the loop against the
    # canonical 124 B per bead-step (mixed) of the integrator's streams
    vv_n, vv_us = kernel_stat(loop_kt, "k_vv_fused")
    pair_n, pair_us_loop = kernel_stat(loop_kt, "k_pair")
    integ = None
    if vv_us:
        integ = {"bound": "hbm", "kernel": "k_vv_fused (verlet_velocities + verlet_positions + check_skin + "
                                           "intra_molec + bending)",
                 "launch_us": vv_us, "launches": vv_n, "algorithmic_bytes": 124 * n,
                 "achieved_gbs": 124 * n / (vv_us * 1e-6) / 1e9,
                 "frac": 124 * n / (vv_us * 1e-6) / 1e9 / hbm_peak,
                 "source": "CUPTI activity records over 200 in-loop steps (L2 warm)"}
    # Ewald k-space (charged workloads): 12 FP64 flops per (charged particle, k)
    # in each of the structure-factor and force passes (canonical count; the
    # neutral particles are not visited)
    ewk = None
    if cfg.params.charged:
        import numpy as np
        nk = int(g.kvecs().shape[0])
        nq = int(np.count_nonzero(cfg.q))
        n_rho, t_rho = kernel_stat(loop_kt, "k_rho_runs")
        if not t_rho:
            n_rho, t_rho = kernel_stat(loop_kt, "k_rho_partial")
        n_red, t_red = kernel_stat(loop_kt, "k_rho_reduce")
        n_ef, t_ef = kernel_stat(loop_kt, "k_force_runs")
        if t_rho and t_ef:
            us = t_rho + (t_red or 0.0) + t_ef
            flops = 2 * 12 * nq * nk
            ewk = {"bound": "fp64 pipe", "k_vectors": nk, "charged_particles": nq, "flops_per_step": flops,
                   "us_per_step": us, "tflops_fp64": flops / (us * 1e-6) / 1e12,
                   "kernels_us": {"structure_factors": t_rho, "k_rho_reduce": t_red, "k_force_runs": t_ef},
                   "peak_note": "no FP64 peak in MEASURED_PEAKS.json; B200's nominal FP64 (non-tensor) rate is "
                                "about 37 TFLOP/s"}
    loop_total = sum(v["total_us"] for v in loop_kt.values())
    loop_share = {short_name(k): round(v["total_us"] / loop_total, 4)
                  for k, v in sorted(loop_kt.items(), key=lambda kv: -kv[1]["total_us"])[:8]} if loop_total else {}
    st_acc = g.download()
    g.close()

    # plain FP64 GPU path, same protocol
    g64, ms_fp64, _, _, s64 = timed_run(_abi.FP64, a.steps, a.warmup)
    g64.close()
    ms_fp64 = max_over_ranks(ms_fp64, dist, f"cuda:{dev}")
    value_fp64 = world * n * a.steps / (ms_fp64 * 1e-3)

    # the mixed path's reported quantities against the FP64 path
    acc = accuracy_vs_fp64(cfg, st_acc, dev) if rank == 0 and a.workload == "brush" else None

    # end to end through the public API with host buffers
    import ctypes as C
    pinned = torch.empty((3, n, 3), dtype=torch.float64, pin_memory=True)
    pinned[0].copy_(torch.from_numpy(cfg.r0))
    pinned[1].copy_(torch.from_numpy(cfg.v))
    ge = System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q, precision=_abi.MIXED, device=dev)
    if cfg.params.charged:
        ge.ewald_k(0)
    ge.init_forces()
    ge.step(a.equil)
    # every step's energies (e_total, v_total, t_fluid: the quantities of
    # fort.60) recorded on the device; each call's entries are copied into
    # pinned host memory behind the call, while the host enqueues the next one
    e2e_calls = [a.chunk] * (a.steps // a.chunk) + ([a.steps % a.chunk] if a.steps % a.chunk else [])
    log_cap = a.steps + 4 * a.chunk + 16
    ge.set_energy_log(1, log_cap)
    # a call's graph is captured on its second call of that length: three
    # untimed calls of each length put the capture before the timed region
    for ln in sorted(set(e2e_calls)):
        for _ in range(3):
            ge.step(ln)
            ge.scalars()
    st = ge.download()
    pinned[0].copy_(torch.from_numpy(st["r0"]))
    pinned[1].copy_(torch.from_numpy(st["v"]))
    pinned[2].copy_(torch.from_numpy(st["a"]))
    host = pinned.numpy()
    pinned_out = torch.empty((2, n, 3), dtype=torch.float64, pin_memory=True).numpy()
    pinned_log = torch.zeros((a.steps, 4), dtype=torch.float64, pin_memory=True).numpy()
    dest = {"r0": pinned_out[0], "v": pinned_out[1]}
    # one untimed round trip through the same pinned buffers: the first DMA
    # from a newly pinned allocation maps it for the device (a one-time cost
    # of the allocation, ~0.6 ms for these 21 MB), as a driver reusing its
    # buffers pays once
    ge.upload(r0=host[0], v=host[1], a=host[2])
    ge.download(_abi.R0 | _abi.V, out=dest)
    ge.sync()
    if dist is not None:
        dist.barrier()
    n_log0 = len(ge.energy_log(log_cap))
    # the timed region starts from an idle device, as a new run does: measured
    # on a B200, the 12.5 MB upload takes ~0.28 ms after 100 ms or more of
    # idle, ~0.85 ms when issued within a few ms of the previous copies or
    # kernels (the untimed round trip just above)
    time.sleep(0.2)
    t0 = time.perf_counter()
    ge.upload(r0=host[0], v=host[1], a=host[2])
    t1 = time.perf_counter()
    done = 0
    for ln in e2e_calls:
        ge.step(ln)                          # mfa_step: `chunk` steps per call, as the timed loop
        # the call's energies, step by step, to the host behind it
        ge.fetch_energy_log(pinned_log[done:], n_log0 + done, ln)
        done += ln
    t2 = time.perf_counter()
    out = ge.download(_abi.R0 | _abi.V, out=dest)   # into pinned host buffers; waits for the steps
    t3 = time.perf_counter()
    sc = ge.scalars()                        # error flags and the last step's energies
    t_e2e = time.perf_counter() - t0
    # wall time of each phase: the upload returns once its copies are done, the
    # step calls return once enqueued, the download waits for the steps and the
    # energy copies queued before it
    e2e_phases = {"upload": round((t1 - t0) * 1e3, 3), "enqueue_steps_and_log_copies": round((t2 - t1) * 1e3, 3),
                  "drain_and_download": round((t3 - t2) * 1e3, 3), "scalars": round((t0 + t_e2e - t3) * 1e3, 3)}
    elog = ge.energy_log(log_cap)
    ge.close()
    assert sc["error_bits"] == 0, "e2e run reported a device error"
    assert len(elog) - n_log0 == a.steps, "energy log: one entry per timed step"
    assert np.array_equal(pinned_log, elog[n_log0:n_log0 + a.steps]), "fetched energies equal the log"
    t_e2e = max_over_ranks(t_e2e, dist, f"cuda:{dev}")
    e2e = world * n * a.steps / t_e2e
    e2e_obj = {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": int(72 * n / a.steps),
               "d2h_bytes_per_step": int(32 + (48 * n + 16 * 8 + 8 * 4) / a.steps),
               "protocol": f"wall clock: state (r0, v, a) uploaded from pinned host memory, {len(e2e_calls)} "
                           f"mfa_step calls of up to {a.chunk} steps, each followed by an asynchronous copy of "
                           "its steps' energies (step, e_total, v_total, t_fluid of every step) into pinned host "
                           "memory, final r0 and v downloaded into pinned host memory (this waits for the steps), "
                           "scalars and error flags read once", "phases_ms": e2e_phases}

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not a.no_cpu:
            rate, steps, dt = run_oracle(cfg, a.cpu_seconds, 100000)
            model, ncpu = cpu_info()
            cpu = {"value": rate, "unit": METRIC, "cores": 1, "kind": "port",
                   "sample": f"{steps} full time steps ({dt:.1f} s) of the same {n}-bead workload, serial C "
                             f"restatement of the reference loop on 1 core of {model} ({ncpu} host threads)"}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator, no reference data)",
            "config": dict(meta, beads=n, precision="mixed", dt=cfg.params.dt, skin=skin_mixed,
                           cells=nbin_mixed, autotune_skin_ms_per_step=skin_tuning,
                           pair_shape=f"{shape_mixed[0]} list entries per thread and round x {shape_mixed[1]}-thread blocks, "
                                      f"{'tiled' if shape_mixed[2] else 'untiled'}"
                                      f"{f', work queue of {shape_mixed[3]} CTAs per SM' if shape_mixed[3] else ''}"
                                      f"{f', each chunk list cut into {shape_mixed[4]} pieces' if shape_mixed[4] > 1 else ''}"
                                      " (autotuned)",
                           autotune_ms_per_step=tuning_mixed,
                           thermostat={_abi.THERMO_DPD: "dpd", _abi.THERMO_LGV: "langevin"}.get(
                               cfg.params.thermostat, "none"), replicas=world,
                           steps_per_timed_iteration=a.chunk,
                           l2=f"flushed between timed iterations of {a.chunk} steps "
                              "(256 MiB write on the context stream)",
                           parallelism=f"replicas x{world}"),
            "fp64": {"value": value_fp64, "ms_per_step": ms_fp64 / a.steps, "per_call_ms": s64["per_call_ms"]},
            "mixed_over_fp64": value / value_fp64,
            "value_l2_resident": world * n * a.steps / (ms_resident * 1e-3),
            "roofline": {"bound": "hbm", "kernel": pair_label,
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": traffic, "traffic_source": traffic_src,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"
                         if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                         "launch_ms": pair_ms, "algorithmic_bytes": pair_bytes,
                         "timing": f"CUDA events around {reps} launches on the context stream, L2 flushed before "
                                   f"every {a.chunk}th as the timed loop flushes it before every call of {a.chunk} steps; "
                                   "a device spin after each flush keeps the host's enqueue ahead of the device",
                         "launch_ms_l2_flushed_each": pair_ms_cold,
                         "launch_us_in_loop": pair_us_loop,
                         "fp32_tflops": pair_flops / (pair_ms * 1e-3) / 1e12,
                         # the FP32 pipe as the pair kernel's other bound: no FP32 peak is
                         # measured, so the fraction is of the nominal non-tensor rate
                         # (148 SMs x 128 lanes x 2 flop x 1.965 GHz)
                         "fp32_frac_of_nominal": pair_flops / (pair_ms * 1e-3) / 74.4e12,
                         "fp32_peak_note": "74.4 TFLOP/s nominal FP32 (non-tensor), not measured", **work},
            "integration": integ,
            "ewald_k": ewk,
            "loop_kernel_share": loop_share,
            "per_call_ms": s_mixed["per_call_ms"],
            "rebuild": {"bound": "hbm", "launch_ms": rebuild_ms, "algorithmic_bytes": 60 * n,
                        "achieved_gbs": 60 * n / (rebuild_ms * 1e-3) / 1e9,
                        "frac": 60 * n / (rebuild_ms * 1e-3) / 1e9 / hbm_peak,
                        "note": "6 kernels (cell assign, row scan, scatter, per-cell sort, gather, list build); "
                                "60 B per bead per rebuild"},
            "e2e": e2e_obj,
            "accuracy_vs_fp64": acc,
            "gpu_launches": int(launches),
            "list_rebuilds_in_timed_steps": int(s_mixed["rebuilds_timed"]),
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
