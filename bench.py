#!/usr/bin/env python
"""Throughput of the CubeSphere per-stage volume update on B200.

One step = one full RK time step (all stages and the CFL reduction) of a
resident solve; the timed steps are replayed from the captured step graph
(cs_steps: time step kept on the device, one host synchronisation at the
end).  The metric is zone-updates/s: interior zones x steps / device
seconds, summed over ranks (each rank runs its own replica of the solve:
one solve is not split across GPUs here).

Default workload ``shell128``: 6 panels x 128^2 angular x 64 radial zones,
radii 1..2 with geometric stretch 1.02, 4 ghost layers, FP64, hydrostatic
1/r^2 shell with seeded density / field perturbations (amplitude 0.05)
under point-mass gravity, IMEX-RK2.  The state (0.8 GB) and the
per-stage work arrays are far larger than L2, so no L2 flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

``--impl reference`` times the CPU oracle port of the same path on the same
workload instead: the oracle builds its own mesh and seeded state (it loads
no other library) and runs one or more whole steps of the full mesh on all
host cores, the timed steps bounded to about a minute and a half.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# Algorithmic DRAM bytes per unit for the kernels that can dominate a stage:
# unique words each kernel must read and write once (state, work arrays and
# geometry it touches), 8 bytes each.  Units: zones of the kernel's range.
ALGO_WORDS_PER_UNIT = {
    # 8 prims x 4 one-sided stencils' neighbours are re-reads; compulsory: 9
    # comps of V/ent mode 1 + 3 centroid + scale + 9 x 3 gradient modes out
    "k_weno7a": 9 + 4 + 27,
    # V modes 0-3 of 8 comps in (32), modes 1-9 out (72), flattener, 10
    # moments, the resident row weights (18 x 9); neighbours' V are re-reads
    "k_weno7b": 32 + 72 + 1 + 10 + 162,
    # resident KKT factors (1296) + pivots (36 bytes) + the 36 right-hand
    # sides in, 30 B modes and U(5:8) out (U read and written: 8)
    "k_adp_solve": 1296 + 4.5 + 36 + 30 + 8,
    # the same with the factors shared by the six panels (1/6 per zone)
    "k_adp_solve6": (1296 + 4.5) / 6 + 36 + 30 + 8,
    # face-B quadrature values (30), B modes (30), geometry of the 6 faces
    # (normals 42, points 90, weights 30) and of the zone (14), 36 out
    "k_adp_rhs": 30 + 30 + 162 + 14 + 36,
    # the same with panel 1's geometry serving the six panels (1/6 per zone)
    "k_adp_rhs6": 30 + 30 + (162 + 14) / 6 + 36,
    # one launch per stage, the three face directions (units = zones): the
    # zone's 80 modes, 4 entropy modes, 10 moments, centroid and scale in;
    # per direction the face geometry (15 points, 5 weights, normals /
    # centroid 6, area, 2 volumes) in and 16 contributions, 2 speeds and the
    # entropy flux out
    "k_flux": 80 + 4 + 10 + 4 + 3 * (15 + 5 + 6 + 1 + 2) + 3 * (16 + 3),
    # E snapshot (3) and modes 1-3 (9) in, E mode 0 out (3), flattener,
    # moments, the resident row weights (19 x 10, panel 1's serving the six
    # panels: 1/6 per zone)
    "k_efield_c": 3 + 9 + 3 + 1 + 10 + 190 / 6,
    "k_positivity": 80 + 4 + 80,
    "k_faceB": 80 + 1 + 20 + 5,
}

# DRAM bytes per unit and launch (read + write) measured by ncu on the
# shell32 case (units: 190,608 zones of the ADP range, 155,520 of the flux /
# least-squares ranges; 14 launches each), FP64 and precision form; the full
# shell128 launches are too large to capture, so roofline.traffic scales
# these by the units of a full launch.
MEASURED_TRAFFIC_PER_UNIT = {
    "k_adp_solve6": 2274.8,
    "k_flux": 2085.8,
    "k_weno7b": 2188.9,
    "k_efield_c": 486.5,
}
MEASURED_TRAFFIC_PER_UNIT_FP32 = {
    "k_adp_solve6": 1117.1,
    "k_flux": 1489.4,
    "k_weno7b": 420.0,
    "k_efield_c": 262.9,
}
# FP64 operations per unit and launch (2 x DFMA + DADD + DMUL thread
# instructions), from the same FP64 capture.  The path is FP64-bound, so the
# roofline also reports these against the FP64 FMA rate measured on the
# device in the same run (cs_fp64_fma_rate); the nominal rate, 148 SMs x 64
# FP64 FMA per clock x 2 x 1.965 GHz = 37.2 TFLOP/s, is kept for context.
FP64_FLOP_PER_UNIT = {
    "k_adp_solve6": 3154.2,
    "k_flux": 16485.3,
    "k_weno7b": 3727.7,
    "k_efield_c": 1529.2,
}
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12

# Compulsory state traffic per zone-update (every stage reads and writes
# the state once, later stages also read the stage-start state; geometry
# and operators re-read are overhead): 12 FP64 words of state per zone in
# the plain form, 9 FP32 + 3 FP64 words (60 B) in the precision form.
#   two stages (RK2, IMEX-RK2): (24 + 36) words = 480 B; FP32 form 300 B
#   SSP-RK3: (24 + 36 + 36) words = 768 B; FP32 form 480 B
def path_bytes_per_zone_update(rk_scheme: int, fp32: bool) -> float:
    state = 60.0 if fp32 else 96.0
    stages = 3 if rk_scheme == 3 else 2
    return state * 2 + state * 3 * (stages - 1)


# Steps after which the precision form's state is compared with the FP64 one.
PRECISION_STEPS = 10

WORKLOAD_DOC = {
    "shell128": "FP64 ideal-MHD hydrostatic shell, 6x128^2x64 zones, r 1..2 stretch 1.02, 4 ghosts, IMEX-RK2, "
                "P12 WENO-AO/MRWENO + ADP, HLL fluxes, LLF multi-D EMFs, CT",
    "shell32": "FP64 ideal-MHD hydrostatic shell, 6x32^2x16 zones, 4 ghosts, IMEX-RK2",
    "surface32": "FP64 ideal-MHD surface, 6x32^2x1 zones, 3 ghosts, SSP-RK3",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cubesphere_b200", choices=["cubesphere_b200", "reference"])
    ap.add_argument("--workload", default="shell128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-form sample")
    ap.add_argument("--no-p2", action="store_true", help="skip the LIMIT_ALL_SLOPES_P2 sample (one GPU only)")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32 precision-form sample")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form sample")
    ap.add_argument("--flags", type=int, default=0,
                    help="cs_params.flags of the timed solve (8: the precision form); the default is the plain FP64 form")
    ap.add_argument("--profile-json", default="", help="also write the per-kernel device times here")
    ap.add_argument("--precision-workload", default="",
                    help="also run the precision form against FP64 over --precision-steps steps of this workload "
                         "(shell256: the 6x256^2x128 statement) and report errors and both forms' times")
    ap.add_argument("--precision-steps", type=int, default=200)
    ap.add_argument("--stated-batch", action="store_true",
                    help="the batched form at its stated size: 64 solves, N in {32..128}, depth in {1..64}")
    ap.add_argument("--stated-serving", action="store_true",
                    help="the serving form at its stated sizes: N in {32..128}, depth in {1..64}, 20-500 steps")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Ranks:
    """Process-group plumbing of a multi-GPU run: every rank times its own
    replica; barrier() lines the ranks up around the timed region and
    allmax() takes the slowest rank's device time (NCCL on the GPUs; the
    same calls work on a gloo group, which the CPU tests use)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist
        self.device = device

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def allmax(self, x: float) -> float:
        if self.dist is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def replica_throughput(zones: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job zone-updates/s: every rank advances its own replica of
    `zones` zones by `steps` steps; the job takes the slowest rank's time."""
    return zones * steps * world / (ms_max / 1e3)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline_sample(name: str, steps: int = 1, warmup: int = 0, budget_s: float = 90.0) -> dict:
    """The oracle (C++ port of the reference CPU path, zone-parallel OpenMP
    on every host core) on the full workload `name`: its own mesh and
    seeded initial state (untimed), `warmup` untimed steps, then whole
    steps timed until `steps` are done or `budget_s` seconds have passed
    (at least one)."""
    threads = host_cores()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import cubesphere_b200 as cs
    from oracle import Oracle

    pr = cs.preset(name)
    t0 = time.perf_counter()
    o = Oracle(params=cs.make_params(**pr["params"]))
    o.init_problem(cs.make_init(**pr["init"]))
    setup = time.perf_counter() - t0
    dt = o.evaluate_timestep(1e30)
    for _ in range(warmup):
        dt = o.step(dt)
    done, sec = 0, 0.0
    while done < max(1, steps):
        t1 = time.perf_counter()
        dt = o.step(dt)
        sec += time.perf_counter() - t1
        done += 1
        if sec >= budget_s:
            break
    o.close()
    p = pr["params"]
    zones = 6 * p["ntp"] ** 2 * p["nr"]
    return {"value": zones * done / sec, "unit": "zone-updates/s", "cores": threads, "kind": "port",
            "sample": f"oracle C++ port (zone-parallel OpenMP, {threads} threads) on the full {name} workload, "
                      f"6x{p['ntp']}^2x{p['nr']} zones: {done} whole step(s) timed ({sec:.1f} s) after {warmup} "
                      f"untimed; mesh + seeded state {setup:.1f} s untimed",
            "steps_timed": done, "seconds": sec}


def serving_sample(seed: int = 7, nreq: int = 24, rate: float = 8.0, max_active: int = 8,
                   sizes=(32, 48, 64), depths=(1, 16, 32), step_range=(20, 60)) -> dict:
    """Serving form: Poisson arrivals (seeded rate) of solve requests with
    panel N from `sizes`, radial depth from `depths` and a step count in
    `step_range`, admitted by free device memory into the concurrent server
    (meshes cached between requests), in the plain FP64 form and in the
    precision form; then the FP64 requests run one at a time (the plain path
    run sequentially, all submitted at once) for the throughput comparison.
    Throughput = zone updates / (last completion - first submission); a
    fresh server per run, so mesh builds are inside.  The defaults are a
    bounded sample; the stated configuration draws N from {32, 48, 64, 96,
    128}, depth from {1, 16, 32, 64} and 20..500 steps."""
    import numpy as np

    import cubesphere_b200 as cs

    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(nreq):
        ntp = int(rng.choice(list(sizes)))
        nr = int(rng.choice(list(depths)))
        steps = int(rng.integers(step_range[0], step_range[1] + 1))
        pr = cs.preset("shell16")
        params = dict(pr["params"])
        init = dict(pr["init"])
        params.update(ntp=ntp, nr=nr, nghost=4 if nr > 1 else 3)
        init.update(seed=int(rng.integers(1, 1 << 30)))
        if nr == 1:
            params.update(gm=0.0, rmin=1.0, rmax=1.05, radial_mesh="uniform", rk_scheme=cs.CS_SSPRK3)
            init.update(kind=0, v_amp=0.5, p0=1.0, rho_amp=0.1, a_amp=0.1)
        reqs.append((steps, params, init))
    gaps = rng.exponential(1.0 / rate, size=nreq)

    def run(max_act, arrivals, flags=0):
        srv = cs.Server(max_active=max_act, mem_fraction=0.8)
        ids = []
        for q, (steps, params, init) in enumerate(reqs):
            if arrivals and q:
                time.sleep(float(gaps[q]))
            ids.append(srv.submit(steps, dict(params, flags=flags), init))
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
        srv.close()
        return {"p50_latency_s": st["p50_s"], "p99_latency_s": st["p99_s"],
                "mean_queue_s": float(np.mean([r.queue_s for r in res])),
                "zone_updates_per_s": st["zone_updates_per_s"],
                "meshes_reused": int(sum(r.mesh_reused for r in res)),
                "all_ok": all(r.status == 0 for r in res)}

    f64 = run(max_active, True)
    f32 = run(max_active, True, cs.CS_FLAG_FP32)
    seq = run(1, False)
    return {"requests": nreq, "arrival_rate_per_s": rate, "max_active": max_active,
            "zone_updates": int(sum(6 * p["ntp"] ** 2 * p["nr"] * n for n, p, _ in reqs)),
            "f64": f64, "f32_precision_form": f32, "f64_sequential": seq,
            "f32_vs_f64_sequential": f32["zone_updates_per_s"] / max(seq["zone_updates_per_s"], 1e-30),
            "sizes": f"N in {set(sizes)}, nr in {set(depths)}, {step_range[0]}-{step_range[1]} steps "
                     "(IMEX-RK2 shells, SSP-RK3 surfaces); latency = submission to completion, mesh builds included"}


def batch_sample(seed: int = 11, nsol: int = 16, steps: int = 4, sizes=(32, 48, 64), depths=(1, 16, 32),
                 mem_fraction: float = 0.85, autotune: bool = True) -> dict:
    """Batched form: nsol independent solves with panel N from `sizes` and
    radial depth from `depths` (seeded; depth 1 is the surface workload,
    SSP-RK3, the others the shell, IMEX-RK2), in the precision form, created
    in draw order while the device's free memory holds them (mem_fraction of
    what was free at the start; solves on equal meshes share one resident
    mesh), advanced together (one graph launch per step, launch shapes
    autotuned per size class) and, for comparison, one after another
    (cs_steps per member), each over `steps` steps, timed by the host clock
    around calls that return after the device work has finished.  The
    defaults are a bounded sample; the stated configuration draws 64 solves
    with N from {32, 48, 64, 96, 128} and depth from {1, 16, 32, 64}."""
    import numpy as np
    import torch

    import cubesphere_b200 as cs

    rng = np.random.default_rng(seed)
    draws = [(int(rng.choice(list(sizes))), int(rng.choice(list(depths))), int(rng.integers(1, 1 << 30)))
             for _ in range(nsol)]
    budget = mem_fraction * torch.cuda.mem_get_info()[0]
    used0 = torch.cuda.mem_get_info()[0]
    sols, meshes, skipped = [], {}, 0
    t_setup = time.perf_counter()
    for ntp, nr, sd in draws:
        pr = cs.preset("shell16")
        params, init = dict(pr["params"]), dict(pr["init"])
        params.update(ntp=ntp, nr=nr, nghost=4 if nr > 1 else 3, flags=cs.CS_FLAG_FP32)
        init.update(seed=sd)
        if nr == 1:
            params.update(gm=0.0, rmin=1.0, rmax=1.05, radial_mesh="uniform", rk_scheme=cs.CS_SSPRK3)
            init.update(kind=0, v_amp=0.5, p0=1.0, rho_amp=0.1, a_amp=0.1)
        need = cs.estimate_device_bytes(**params)
        if (used0 - torch.cuda.mem_get_info()[0]) + need > budget:
            skipped += 1  # the device is full: the solve is not admitted to this batch
            continue
        s = cs.Solve(**params)
        if (ntp, nr) in meshes:
            s.mesh_share(meshes[(ntp, nr)])
        else:
            s.mesh_build()
            meshes[(ntp, nr)] = s
        s.init_problem(**init)
        sols.append(s)
    t_setup = time.perf_counter() - t_setup
    zones = sum(6 * s.N * s.N * s.nr for s in sols)
    dts = [s.evaluate_timestep(1e30) for s in sols]
    b = cs.Batch(sols)
    t_tune = time.perf_counter()
    if autotune:
        b.autotune(1)
    t_tune = time.perf_counter() - t_tune
    fr = sorted({b.grid_fraction(q) for q in range(len(sols))})
    dts = b.steps(1, dts)  # warm-up: builds the batch graph
    torch.cuda.synchronize()
    # every call below returns after reading the members' next time steps,
    # i.e. after their device work has finished
    t0 = time.perf_counter()
    dts = b.steps(steps, dts)
    bat_s = time.perf_counter() - t0
    b.close()
    t0 = time.perf_counter()
    dts = [s.steps(steps, d) for s, d in zip(sols, dts)]  # one member after another
    seq_s = time.perf_counter() - t0
    ok = all(np.isfinite(d) and d > 0 for d in dts)
    for s in sols:
        s.close()
    return {"solves_drawn": nsol, "solves": len(sols), "not_admitted": skipped, "zones": zones, "steps": steps,
            "dtype": "f32 bulk (precision form)",
            "batched_zone_updates_per_s": zones * steps / bat_s,
            "sequential_zone_updates_per_s": zones * steps / seq_s,
            "setup_s": t_setup, "autotune_s": t_tune, "grid_fractions_chosen": fr, "distinct_meshes": len(meshes),
            "finite": ok,
            "sizes": f"N in {set(sizes)}, nr in {set(depths)}; host wall clock around the device-synchronised runs"}


def precision_sample(pr, dts, steps, ref_state, zones, world, allmax) -> dict:
    """The precision form (CS_FLAG_FP32) on the same workload: from the same
    initial state with the same time steps as the FP64 run (`dts`), the
    relative L1 / Linf errors of its state against the FP64 state after
    those steps (interior zones; faces for B) and its max |div B|; then
    `steps` further steps timed with CUDA events as in the FP64 timing."""
    import torch

    import cubesphere_b200 as cs

    f = cs.Solve(**pr["params"], flags=cs.CS_FLAG_FP32)
    f.mesh_build()
    f.init_problem(**pr["init"])
    stream = torch.cuda.ExternalStream(f.stream_ptr())
    f.evaluate_timestep(1e30)
    dt = dts[0]
    for d in dts:
        dt = f.step(d)
    got = f.get_state()
    _, _, divb = f.diag()
    f.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    f.steps(steps, dt)
    e1.record(stream)
    e1.synchronize()
    ms = allmax(e0.elapsed_time(e1))
    err, err_inf, divb_rel = state_errors(f, got, ref_state, divb)
    f.close()
    return {"value": zones * steps * world / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / steps,
            "dtype": "f32 state/reconstruction/fluxes/least-squares inverses, f64 face B/ADP/EMFs/geometry",
            "steps_compared": len(dts), "l1_rel_err_vs_f64": err, "linf_rel_err_vs_f64": err_inf,
            "max_divb_over_bmax": divb_rel, "long_run": precision_long_sample()}


def p2_sample(pr, steps: int, zones: int) -> dict:
    """LIMIT_ALL_SLOPES_P2 (CS_FLAG_P2) in place of P12 on the same workload
    and precision: 3 untimed steps, then `steps` steps replayed from the
    captured step graph and timed with CUDA events as the headline."""
    import torch

    import cubesphere_b200 as cs

    f = cs.Solve(**pr["params"], flags=cs.CS_FLAG_P2)
    f.mesh_build()
    f.init_problem(**pr["init"])
    stream = torch.cuda.ExternalStream(f.stream_ptr())
    dt = f.steps(3, f.evaluate_timestep(1e30))
    f.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dt = f.steps(steps, dt)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    _, _, divb = f.diag()
    f.close()
    return {"value": zones * steps / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / steps,
            "reconstruction": "LIMIT_ALL_SLOPES_P2 (420limit_all_slopes_p2.f): eight one-sided quadratic stencils "
                              "+ the central least squares, resident stencil inverses",
            "finite": bool(dt == dt and dt > 0), "max_divb": divb}


def state_errors(s, got, ref, divb):
    """Relative L1 and Linf errors of `got` against `ref` per field (interior
    zones; the three face-B components as one field) and max |div B| over
    max |B|."""
    import numpy as np

    G, N, nr = s.G, s.N, s.nr
    I = s.interior

    def l1(a, b):
        return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))

    def linf(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

    def fc(a, d):
        lo = [1, 1, 1]
        lo[d] = 0
        return a[..., G + lo[2]:G + nr + 1, G + lo[1]:G + N + 1, G + lo[0]:G + N + 1]

    fields = {"rho": (I(got["U"][0]), I(ref["U"][0])), "momentum": (I(got["U"][1:4]), I(ref["U"][1:4])),
              "energy": (I(got["U"][4]), I(ref["U"][4])), "entropy": (I(got["ent"]), I(ref["ent"])),
              "face_B": (np.concatenate([fc(got[k], d).ravel() for d, k in enumerate(("bxf", "byf", "bzf"))]),
                         np.concatenate([fc(ref[k], d).ravel() for d, k in enumerate(("bxf", "byf", "bzf"))]))}
    bmax = float(np.abs(fc(got["bxf"], 0)).max())
    return ({k: l1(*v) for k, v in fields.items()}, {k: linf(*v) for k, v in fields.items()}, float(divb) / bmax)


def precision_long_sample(name: str = "shell32", nsteps: int = 200, timed: bool = False) -> dict:
    """The precision form over a long run: the FP64 form first (its time
    step of every step recorded, its final state kept on the host, its
    device freed), then the precision form from the same initial state with
    the same time steps; relative L1 / Linf errors and max |div B| after
    `nsteps` steps.  The FP64 run drops the resident operators
    (CS_FLAG_NO_ADP_CACHE | CS_FLAG_NO_OP_CACHE: the same results to
    round-off) when the device cannot hold them, as on the 6 x 256^2 x 128
    shell, where the precision form drops the least-squares row weights
    (CS_FLAG_NO_OP_CACHE) to keep its ADP factors.  With `timed`, each run's device time per step (CUDA events
    around the step loop, one host read of the time step per step)."""
    import torch

    import cubesphere_b200 as cs

    pr = cs.preset(name)
    free = torch.cuda.mem_get_info()[0]
    f64_flags = 0
    if cs.estimate_device_bytes(**pr["params"]) > 0.9 * free:
        f64_flags = cs.CS_FLAG_NO_ADP_CACHE | cs.CS_FLAG_NO_OP_CACHE

    def run(flags, dts_in):
        s = cs.Solve(**pr["params"], flags=flags)
        s.mesh_build()
        s.init_problem(**pr["init"])
        dt = s.evaluate_timestep(1e30)
        dts = []
        stream = torch.cuda.ExternalStream(s.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.synchronize()
        e0.record(stream)
        t0 = time.time()
        for n in range(nsteps):
            d = dts_in[n] if dts_in is not None else dt
            dts.append(d)
            dt = s.step(d)
            if nsteps >= 50 and (n + 1) % 25 == 0:
                print(f"precision run flags={flags}: step {n + 1}/{nsteps}, {time.time() - t0:.0f} s", file=sys.stderr,
                      flush=True)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / nsteps
        got = s.get_state()
        _, _, divb = s.diag()
        s.close()
        return got, dts, divb, ms

    ref, dts, _, ms64 = run(f64_flags, None)
    torch.cuda.synchronize()
    # the precision form keeps its ADP factors (the costly rebuild) and drops
    # the cheaper least-squares row weights when the device cannot hold both
    f32_flags = cs.CS_FLAG_FP32
    if cs.estimate_device_bytes(**dict(pr["params"], flags=f32_flags)) > 0.9 * torch.cuda.mem_get_info()[0]:
        f32_flags |= cs.CS_FLAG_NO_OP_CACHE
    got, _, divb, ms32 = run(f32_flags, dts)
    shape = cs.Solve(**pr["params"])
    err, err_inf, divb_rel = state_errors(shape, got, ref, divb)
    shape.close()
    p = pr["params"]
    out = {"workload": name, "zones": 6 * p["ntp"] ** 2 * p["nr"], "steps_compared": nsteps,
           "l1_rel_err_vs_f64": err, "linf_rel_err_vs_f64": err_inf, "max_divb_over_bmax": divb_rel,
           "f64_flags": f64_flags, "f32_flags": f32_flags}
    if timed:
        zones = out["zones"]
        out.update({"f64_ms_per_step": ms64, "f32_ms_per_step": ms32,
                    "f64_zone_updates_per_s": zones / (ms64 / 1e3), "f32_zone_updates_per_s": zones / (ms32 / 1e3),
                    "timing": "CUDA events around each run's step loop (one host read of the time step per step)"})
    return out


def workload_config(args, zones: int, world: int) -> dict:
    import cubesphere_b200 as cs

    return {"workload": args.workload, "desc": WORKLOAD_DOC.get(args.workload, ""), "flags": args.flags,
            "zones": zones, "parallelism": f"replicas x{world}",
            "precision": "f32 bulk / f64 B" if args.flags & cs.CS_FLAG_FP32 else "f64",
            "reconstruction": "LIMIT_ALL_SLOPES_P2" if args.flags & cs.CS_FLAG_P2 else "LIMIT_ALL_SLOPES_P12",
            "l2": "inputs larger than L2 (state and work arrays >> 126 MB), no flush"}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    import cubesphere_b200 as cs

    p = cs.preset(args.workload)["params"]
    zones = 6 * p["ntp"] ** 2 * p["nr"]
    r = cpu_baseline_sample(args.workload, steps=args.steps, warmup=min(args.warmup, 1))
    v = r["value"]
    out = {
        "metric": "zone-updates/s", "value": v, "unit": "zone-updates/s", "n_gpus": args.gpus,
        "steps": r["steps_timed"], "warmup": min(args.warmup, 1), "ms_per_step": r["seconds"] * 1e3 / r["steps_timed"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded harmonic density / vector-potential perturbations)",
        "config": workload_config(args, zones, world),
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": r["cores"], "kind": "port",
                         "sample": r["sample"]},
        "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


def run_gpu(args):
    import numpy as np
    import torch

    import cubesphere_b200 as cs

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    ranks = Ranks(dist, "cuda")
    barrier, allmax = ranks.barrier, ranks.allmax

    pr = cs.preset(args.workload)
    s = cs.Solve(**pr["params"], flags=args.flags)
    s.mesh_build()
    s.init_problem(**pr["init"])
    zones = 6 * s.N * s.N * s.nr
    stream = torch.cuda.ExternalStream(s.stream_ptr())
    dt = s.evaluate_timestep(1e30)
    dts = []  # the time step of every step from the initial state
    for _ in range(max(args.warmup, 3)):
        dts.append(dt)
        dt = s.step(dt)
    # the precision form is compared with this state after PRECISION_STEPS
    # steps of known time step (untimed)
    ref_state = None
    if not (args.no_precision or args.flags):
        while len(dts) < PRECISION_STEPS:
            dts.append(dt)
            dt = s.step(dt)
        ref_state = s.get_state()
    s.steps(1, dt)  # captures the step graph before the timed region

    # ---- device-resident timing: args.steps steps replayed from the
    # captured step graph (device-resident time step, one host
    # synchronisation at the end)
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    s.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = s.launch_count()
    clocks.start()
    e0.record(stream)
    dt = s.steps(args.steps, dt)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    launches = s.launch_count() - l0
    ms = allmax(e0.elapsed_time(e1))
    barrier()
    value = replica_throughput(zones, args.steps, world, ms)

    # ---- per-kernel device times: one more step with events between the
    # launches (untimed; feeds top_kernels and the roofline)
    s.profile_begin()
    dt = s.step(dt)
    prof = s.profile_end()
    prof_steps = 1

    # ---- end to end through the C ABI with pinned host buffers
    host = {}
    for k in ("U", "ent", "bxf", "byf", "bzf"):
        nc = 8 if k == "U" else 1
        host[k] = torch.empty(s.shape(nc), dtype=torch.float64, pin_memory=True).numpy()
    s.get_state(host)
    h2d = sum(a.nbytes for a in host.values())
    d2h = h2d
    barrier()
    torch.cuda.synchronize()
    s.synchronize()
    k_e2e = max(1, min(args.steps, 5))
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        s.put_state(host)
        dt = s.step(dt)
        s.get_state(host)
    f1.record(stream)
    f1.synchronize()
    ms_e2e = allmax(f0.elapsed_time(f1))
    e2e = replica_throughput(zones, k_e2e, world, ms_e2e)
    finite = bool(np.isfinite(host["U"]).all())

    # ---- roofline of the dominant kernel (by device time in the timed region)
    import json as _json

    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = _json.loads(pk.read_text())
    hbm_peak = None
    peak_note = "measured"
    for key in ("hbm_gbs", "hbm_GBs", "hbm_gb_s"):
        if key in peaks:
            hbm_peak = float(peaks[key])
    if hbm_peak is None:
        hbm_peak, peak_note = 6650.0, "fallback"
    # Algorithmic bytes of the path (compulsory state traffic per
    # zone-update); the dominant kernel is charged one stage's share of them
    # for the zones one launch covers, and its own read/write set and its
    # measured DRAM traffic are reported beside that.
    fp32 = bool(args.flags & cs.CS_FLAG_FP32)
    rk = int(pr["params"]["rk_scheme"])
    path_b = path_bytes_per_zone_update(rk, fp32)
    stage_b = path_b / (3 if rk == 3 else 2)
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dname, (dms, dcount) = dom
    G, N, nr = s.G, s.N, s.nr
    units = 6 * (N + 2 * G - 2) ** 2 * (nr + 2 * G - 2)  # zones of the shrink-1 range (7.a / 8.d / 9.b)
    if dname in ("k_weno7b", "k_efield_c"):
        units = 6 * (N + 2 * G - 4) ** 2 * (nr + 2 * G - 4)
    if dname == "k_flux":
        units = 6 * (N + 4) ** 2 * (nr + 4)
    launch_s = dms / dcount / 1e3
    per_launch = stage_b * units
    achieved = per_launch / launch_s / 1e9
    tr = (MEASURED_TRAFFIC_PER_UNIT_FP32 if fp32 else MEASURED_TRAFFIC_PER_UNIT).get(dname)
    traffic = tr * units if tr else None
    words = ALGO_WORDS_PER_UNIT.get(dname)
    per_value = value / world  # one GPU's zone-updates/s
    roof = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_note + " (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_unit": stage_b,
            "unit_def": f"zone-stage: {path_b:.0f} B per zone-update / {3 if rk == 3 else 2} stages; "
                        f"{units} zones per launch",
            "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": dms / dcount,
            "share_of_step": dms / sum(v[0] for v in prof.values()),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum on shell32, scaled by units"
            if tr else None,
            "dram_frac": (traffic / launch_s / 1e9 / hbm_peak) if traffic else None,
            "traffic_ratio": (traffic / per_launch) if traffic else None,
            "kernel_read_write_bytes_per_launch": (words * 8.0 * units) if words else None,
            "path": {"bytes_per_zone_update": path_b, "achieved_gbs": path_b * per_value / 1e9,
                     "frac": path_b * per_value / 1e9 / hbm_peak}}
    fp64_peak = None
    try:
        fp64_peak = cs.fp64_fma_rate(16384)
    except cs.CsError:
        pass
    fl = FP64_FLOP_PER_UNIT.get(dname)
    if fl and not fp32:
        tf = fl * units / launch_s / 1e12
        den = fp64_peak or FP64_NOMINAL_TFLOPS
        roof["fp64"] = {"achieved_tflops": tf, "peak_tflops": den, "frac": tf / den,
                        "peak_source": "measured DFMA chains on this device (cs_fp64_fma_rate)" if fp64_peak
                        else "nominal (148 SMs x 64 FMA/clk x 2 x 1.965 GHz)",
                        "nominal_tflops": FP64_NOMINAL_TFLOPS,
                        "flop_per_unit_source": "ncu DFMA/DADD/DMUL counts on shell32"}

    s.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args.workload, steps=1, warmup=0, budget_s=60.0)
    precision = None
    if ref_state is not None:
        torch.cuda.synchronize()
        precision = precision_sample(pr, dts[:PRECISION_STEPS], args.steps, ref_state, zones, world, allmax)
    p2 = None
    if world == 1 and not (args.no_p2 or args.flags):
        torch.cuda.synchronize()
        try:
            p2 = p2_sample(pr, args.steps, zones)
        except Exception as e:  # recorded, not fatal: the headline line still prints
            p2 = {"error": f"{type(e).__name__}: {e}"}
    precision_stated = None
    if args.precision_workload:
        torch.cuda.synchronize()
        precision_stated = precision_long_sample(args.precision_workload, args.precision_steps, timed=True)
    batch = None
    if args.stated_batch:
        torch.cuda.synchronize()
        batch = batch_sample(seed=11, nsol=64, steps=2, sizes=(32, 48, 64, 96, 128), depths=(1, 16, 32, 64))
    elif not args.no_batch and world == 1:  # single-GPU characterisations: not repeated on every rank
        torch.cuda.synchronize()
        batch = batch_sample()
    serving = None
    if args.stated_serving:
        torch.cuda.synchronize()
        serving = serving_sample(seed=7, nreq=24, rate=2.0, max_active=8, sizes=(32, 48, 64, 96, 128),
                                 depths=(1, 16, 32, 64), step_range=(20, 500))
    elif not args.no_serving and world == 1:
        torch.cuda.synchronize()
        serving = serving_sample()

    if args.profile_json and rank == 0:
        Path(args.profile_json).write_text(_json.dumps(
            {k: {"ms": v[0], "launches": v[1]} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
            indent=1))

    out = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 bulk / f64 B" if args.flags & cs.CS_FLAG_FP32 else "f64",
        "data": "synthetic (seeded harmonic density / vector-potential perturbations)",
        "config": workload_config(args, zones, world),
        "e2e": {"value": e2e, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": k_e2e},
        "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
        "top_kernels": {k: round(v[0] / prof_steps, 3) for k, v in
                        sorted(prof.items(), key=lambda kv: -kv[1][0])[:8]},
        "finite": finite, "dt_last": dt, "precision_form": precision, "p2_form": p2, "precision_stated": precision_stated,
        "batch": batch, "serving": serving,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    raise SystemExit(main())
