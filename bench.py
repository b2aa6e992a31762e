#!/usr/bin/env python
"""Benchmark: FP64 cell-updates/s of the SSP-RK2 shallow-water step.

Workload (N = 1): 2048 x 2048 Cartesian cells, dx = 2 m, FP64: wet/dry dam
break over a seeded sloping beach (1:50 plus 0.3 m smooth noise), dry land
initially, Manning n = 0.03, Flather open boundary on the west side, walls
elsewhere; each step takes dt = maxDt() (CFL 0.45).  One "step" is one full
SSP-RK2 step of the whole grid: 2048 * 2048 cell-updates.  The device holds
b, two copies of (h, hu, hv) and the metric, about 236 MB -- larger than the
126 MB L2, so nothing is flushed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun, one process per GPU): every rank advances its own
independent basin of the same size (weak scaling, no data-path collective);
the timed region is bracketed by a barrier and the max over ranks is taken.

--impl reference times the CPU restatement of the reference solver (the
oracle; the reference itself is JavaScript and no JS engine exists on the
box) with every host thread, on a bounded sample of the same workload.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 2048
DX = 2.0
MANNING = 0.03
METRIC = "FP64 cell-updates/s"
UNIT = "cell-updates/s"
STAGE_BYTES = {"stage1": 56, "stage2": 80}      # algorithmic HBM bytes per cell per launch
STEP_BYTES = 136                                # per cell-update (both stages)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="leave out the all-wet, batched-ensemble and adjoint objects of the 1-GPU line")
    p.add_argument("--workload", default="beach",
                   choices=["beach", "ensemble", "adjoint", "sphere", "slabs", "allwet"],
                   help="beach: the 2048x2048 headline; ensemble: the 256-basin batched form vs the plain "
                        "kernel; sphere: the 1440x720 tide; adjoint: the 1024x1024 misfit gradient; slabs: "
                        "the beach cut into row slabs over the ranks (device halo exchange)")
    p.add_argument("--stage", default="default", choices=["default", "fused", "split"],
                   help="stage kernels: the library default, the fused row-marching kernel or the tiled pair")
    p.add_argument("--nx", type=int, default=2048, help="grid size (the workload is 2048x2048)")
    p.add_argument("--ny", type=int, default=2048)
    a = p.parse_args()
    global NX, NY
    NX, NY = a.nx, a.ny
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload():
    import __graft_entry__
    swe = __graft_entry__.load_package()
    from water_simulator_b200.workloads import beach_dam_break
    b, eta = beach_dam_break(NX, NY, DX)
    return swe, b, eta


def config(extra=None):
    c = {"workload": "cartesian 2048x2048 dx=2 m wet/dry dam break over a seeded 1:50 beach, "
                     "Manning 0.03, Flather west, dt = maxDt()",
         "nx": NX, "ny": NY, "cells_per_step": NX * NY, "l2": "inputs larger than L2 (236 MB resident)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_figure(name, key):
    """A number recorded in a committed ncu summary under profiles/ (a line
    `key value ...`), or None."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith(key):
                try:
                    return float(line[len(key):].split()[0])
                except (ValueError, IndexError):
                    return None
    return None


def profile_traffic(impl):
    """Per-launch DRAM bytes of stage 2 from the committed ncu summary of the
    stage kernels in use (the tiled pair, or the fused kernel)."""
    name = "k_split_stage_beach2048.md" if impl == 1 else "k_stage2_beach2048.md"
    return profile_figure(name, "dram_bytes_per_launch_full_size:")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.proc = None
        self.gpu = gpu_index
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(gpu_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_oracle_sim(b, eta, threads):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_sim import OracleSim
    sim = OracleSim(nx=NX, ny=NY, dx=DX, bed=b, eta0=eta, manning=MANNING, threads=threads)
    sim.set_boundaries(west=("flather", lambda t: 0.0, lambda t: 0.0), east="reflect",
                       south="reflect", north="reflect")
    return sim


def cpu_baseline(b, eta, threads=1, budget_s=12.0, max_steps=30):
    """The oracle on the host cores: steps of the same workload until the
    time budget is used (at least one)."""
    sim = cpu_oracle_sim(b, eta, threads)
    sim.step()                      # warm (first touch)
    n, t0 = 0, time.perf_counter()
    while True:
        sim.step()
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= max_steps:
            break
    return {"value": NX * NY * n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} self-timed steps of the 2048x2048 workload ({el:.1f} s) on the oracle "
                      f"(C++ restatement of src/swe.mjs), {threads} thread(s)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    _, b, eta = workload()
    threads = os.cpu_count() or 1
    sim = cpu_oracle_sim(b, eta, threads)
    for _ in range(max(args.warmup, 0)):
        sim.step()
    steps = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step()
    el = time.perf_counter() - t0
    v = NX * NY * steps / el
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config({"threads": threads}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} self-timed steps of the 2048x2048 workload on the oracle "
                                       f"(C++ restatement of src/swe.mjs; the reference is JavaScript and "
                                       f"no JS engine exists here), {threads} OpenMP threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def make_sim(swe, b, eta):
    """The beach with Flather(eta_ext = 0, u_ext = 0) on the west side, given
    as a tide of no constituents at msl 0, which the device evaluates inside
    its own loop (so `run` stays one CUDA graph replay per 32 steps)."""
    sim = swe.ShallowWater(nx=NX, ny=NY, dx=DX, bed=b, eta0=eta, manning=MANNING)
    sim.boundaries = {"west": swe.flather(swe.Tide({}, msl=0.0).signal()), "east": swe.reflect,
                      "south": swe.reflect, "north": swe.reflect}
    return sim


def timed_on(torch, stream_ptr, fn, device=0):
    """fn() bracketed by CUDA events on the library's stream (and clocks
    sampled meanwhile): (result, ms, clocks)."""
    st = torch.cuda.ExternalStream(stream_ptr, device=torch.device("cuda", device))
    torch.cuda.synchronize()
    sampler = ClockSampler(device)
    time.sleep(0.25)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    out = fn()
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1), sampler.stop()


def stream_of(swe, sim):
    sp = ctypes.c_void_p()
    swe._lib.check(swe.load_library().swe_get_stream(sim._h, ctypes.byref(sp)))
    return sp.value


def all_wet_summary(torch, swe, steps, device=0, warm=32):
    """An all-wet 2048 x 2048 grid (bump + roughness bed, dam break 3.0 /
    2.5 m, Manning 0.03, walls): every tile computes every cell, so this is
    the rate of the wet-cell kernels, with the roofline of the stage-2 pair."""
    from water_simulator_b200.workloads import bump_bed, _centres
    n = 2048
    b = bump_bed(n, n, DX)
    X, _ = _centres(n, n, DX)
    eta = np.where(X < n * DX / 2, 3.0, 2.5)
    sim = swe.ShallowWater(nx=n, ny=n, dx=DX, bed=b, eta0=eta, manning=MANNING)
    sim.run(warm)
    sim.synchronize()
    done, ms, clocks = timed_on(torch, stream_of(swe, sim), lambda: sim.run(steps), device)
    if done != steps:
        raise RuntimeError(f"all-wet: the device loop took {done} of {steps} steps")
    lib = swe.load_library()
    msv = (ctypes.c_double * 5)()
    dt = sim.maxDt()
    ph = []
    for _ in range(12):
        swe._lib.check(lib.swe_step_timed(sim._h, dt, msv))
        ph.append(list(msv))
    avg = [statistics.mean(p[q] for p in ph[2:]) for q in range(5)]
    dry = int(np.count_nonzero(np.asarray(sim.field("h")).reshape(n + 4, n + 4)[2:-2, 2:-2] <= 1e-3))
    sim.close()
    peak, kind = measured_peaks()
    st2 = STAGE_BYTES["stage2"] * n * n / (avg[4] / 1e3) / 1e9
    return {"workload": "cartesian 2048x2048 dx=2 m, bump+roughness bed, dam break 3.0/2.5 m (every cell wet), "
                        "Manning 0.03, walls, dt = maxDt()",
            "value": n * n * steps / (ms / 1e3), "unit": UNIT, "steps": steps, "ms_per_step": ms / steps,
            "dry_cells_after": dry,
            "step_phase_ms": dict(zip(["prepare", "bc1", "stage1", "bc2", "stage2"], avg)),
            "roofline": {"bound": "hbm", "limiter": "the FP64 pipe (fp64_ceiling)",
                         "achieved": st2, "peak": peak, "unit": "GB/s", "frac": st2 / peak,
                         "peak_source": kind, "algorithmic_bytes_per_launch": STAGE_BYTES["stage2"] * n * n,
                         "traffic": profile_figure(ALLWET_PROFILE, "dram_bytes_per_stage2_pair:")},
            "fp64_ceiling": fp64_ceiling(n * n * steps / (ms / 1e3), peak),
            "clocks": clocks}


ALLWET_PROFILE = "k_split_faces_allwet2048.md"


def fp64_ceiling(cups, peak):
    """What the FP64 pipe allows on the all-wet grid, from the committed ncu
    capture of the stage-2 pair: each kernel's duration times the share of
    it the FP64 pipe was busy is the time its FP64 work needs at full pipe
    rate; the rate with every stage at that bound, against the rate that 60%
    of HBM bandwidth would give at 136 B per cell-update."""
    f = {k: profile_figure(ALLWET_PROFILE, k + ":") for k in
         ("fp64_pipe_active_frac_faces", "fp64_pipe_active_frac_cells", "ncu_us_faces", "ncu_us_cells")}
    if any(v is None for v in f.values()):
        return None
    pair = f["ncu_us_faces"] + f["ncu_us_cells"]
    floor = f["fp64_pipe_active_frac_faces"] * f["ncu_us_faces"] + f["fp64_pipe_active_frac_cells"] * f["ncu_us_cells"]
    return {"fp64_pipe_active_frac": {"faces": f["fp64_pipe_active_frac_faces"], "cells": f["fp64_pipe_active_frac_cells"]},
            "stage2_pair_us": pair, "stage2_fp64_bound_us": floor,
            "cups_at_fp64_bound": cups * pair / floor,
            "cups_at_60pct_hbm": 0.6 * peak * 1e9 / (STAGE_BYTES["stage1"] + STAGE_BYTES["stage2"]),
            "source": "profiles/" + ALLWET_PROFILE}


def ensemble_summary(torch, swe, steps=200, fused_steps=50, device=0):
    """The 256-basin ensemble advanced batched against the plain
    single-grid kernels run basin by basin (each basin through its own
    device loop, device times summed), for both plain stage kernels."""
    from water_simulator_b200 import workloads
    bs = workloads.ensemble()
    cells = sum(b["nx"] * b["ny"] for b in bs)
    ens = swe.Ensemble(bs)
    tuned = ens.autotune(trial_steps=3)
    ens.run(16)
    ens.synchronize()
    _, ms_b, clocks = timed_on(torch, ens.stream(), lambda: ens.run(steps), device)
    ens.close()

    def plain(stage, k):
        total = 0.0
        for b in bs:
            sim = swe.ShallowWater(nx=b["nx"], ny=b["ny"], dx=b["dx"], bed=b["b"], eta0=b["eta0"],
                                   manning=b["manning"])
            if stage == "fused":
                swe._lib.check(swe.load_library().swe_set_stage_kernels(sim._h, 0))
            t = b["tide"]
            tide = swe.Tide({"X": [t["amp"][0], t["phase_deg"][0]]}, msl=t["msl"],
                            periods_hours={"X": 2 * math.pi / t["omega"][0] / 3600})
            tide.terms[0]["omega"] = t["omega"][0]
            sim.boundaries = {"west": swe.flather(tide.signal())}
            sim.run(4)
            done, ms, _ = timed_on(torch, stream_of(swe, sim), lambda: sim.run(k), device)
            assert done == k
            total += ms
            sim.close()
        return cells * k / (total / 1e3), total / k

    tiled, tiled_ms = plain("split", steps)
    fused, fused_ms = plain("fused", fused_steps)
    batched = cells * steps / (ms_b / 1e3)
    return {"workload": "256 Cartesian basins, nx~U[64,1024], ny~U[64,512], dx 5 m, bump+roughness beds, still "
                        "2 m, Manning~U[0.015,0.04], west Flather tide 0.5 m, period~U[2,14] h",
            "cells": cells, "value": batched, "unit": UNIT, "steps": steps, "ms_per_step": ms_b / steps,
            "schedule": tuned,
            "plain_tiled_per_basin": {"value": tiled, "ms_per_step": tiled_ms, "steps": steps,
                                      "how": "the default tiled stage pair, swe_run per basin, device time summed"},
            "plain_fused_per_basin": {"value": fused, "ms_per_step": fused_ms, "steps": fused_steps,
                                      "how": "the fused row-marching stage kernel, swe_run per basin, device "
                                             "time summed"},
            "batched_over_plain_tiled": batched / tiled, "batched_over_plain_fused": batched / fused,
            "clocks": clocks}


def adjoint_summary(torch, swe, steps=180, n=1024, device=0):
    """One gradient of the gauge misfit on the 1024 x 1024 case (recording
    forward + backward with a checkpoint every 45 steps) against the plain
    forward of the same steps, at a reduced step count."""
    from water_simulator_b200 import workloads
    c = workloads.adjoint_case(nx=n, ny=n, dx=10.0, n_gauges=32)
    kw = dict(manning_field=c["n"], gauges=c["gauges"], steps=steps, checkpoint_every=45)
    truth = swe.MisfitAdjoint(n, n, 10.0, c["b_true"], c["eta0"], **kw)
    _, obs = truth.forward()
    truth.close()
    sim = swe.ShallowWater(nx=n, ny=n, dx=10.0, bed=c["b"], eta0=c["eta0"])
    sim.setManningField(c["n"])
    sim.run(steps)
    sim.close()
    sim = swe.ShallowWater(nx=n, ny=n, dx=10.0, bed=c["b"], eta0=c["eta0"])
    sim.setManningField(c["n"])
    sim.synchronize()
    _, t_plain, clocks = timed_on(torch, stream_of(swe, sim), lambda: sim.run(steps), device)
    sim.close()
    adj = swe.MisfitAdjoint(n, n, 10.0, c["b"], c["eta0"], **kw)
    adj.set_observations(obs)
    adj.forward()
    adj.backward()                         # warm-up gradient (the tape is allocated here)
    (J, _), t_fwd, _ = timed_on(torch, adj.stream(), adj.forward, device)
    _, t_bwd, _ = timed_on(torch, adj.stream(), adj.backward, device)
    adj.close()
    return {"workload": f"{n}x{n} dx=10 m, bump+roughness bed, 0.5 m released hump over 2 m still water, Manning "
                        f"field U[0.015,0.04], 32 gauges, checkpoint every 45 steps, {steps} steps (of the "
                        "configuration's 2000)",
            "value": (t_fwd + t_bwd) / t_plain, "unit": "x forward", "higher_is_better": False,
            "steps": steps, "forward_plain_ms": t_plain, "forward_recording_ms": t_fwd, "backward_ms": t_bwd,
            "J": J, "clocks": clocks}


def run_ours(args):
    rank, world, local = dist_env()
    import torch
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    swe, b, eta = workload()
    lib = swe.load_library()
    swe._lib.check(lib.swe_set_device(local))
    sim = make_sim(swe, b, eta)
    stream_ptr = ctypes.c_void_p()
    swe._lib.check(lib.swe_get_stream(sim._h, ctypes.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=torch.device("cuda", local))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up: W steps through the device loop (also builds the CUDA graph)
    sim.run(max(args.warmup, 3))
    sim.synchronize()
    K = args.steps
    sim.run(min(K, 32))             # same graph shape as the timed loop
    sim.synchronize()

    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = sim.run(K)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    barrier()
    if done != K:
        raise RuntimeError(f"the device loop took {done} of {K} steps")
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * NX * NY * K / (ms_max / 1e3)

    # per-launch durations (events between launches on the library's stream)
    dt = sim.maxDt()
    phases = {"prepare": [], "bc1": [], "stage1": [], "bc2": [], "stage2": []}
    msv = (ctypes.c_double * 5)()
    for _ in range(20):
        swe._lib.check(lib.swe_step_timed(sim._h, dt, msv))
        for key, v in zip(phases, msv):
            phases[key].append(v)
    avg = {k: statistics.mean(v[2:]) for k, v in phases.items()}
    step_ms = sum(avg.values())
    peak, peak_kind = measured_peaks()
    st2_bytes = STAGE_BYTES["stage2"] * NX * NY
    achieved = st2_bytes / (avg["stage2"] / 1e3) / 1e9
    impl = ctypes.c_int(-1)
    swe._lib.check(lib.swe_get_stage_kernels(sim._h, ctypes.byref(impl)))
    traffic = profile_traffic(impl.value)
    kname = ("k_split_faces + k_split_cells<2> (stage 2: faces, then limiter + gather + update + friction + "
             "sponge + CFL epilogue)" if impl.value == 1 else
             "k_stage<2> (stage 2 + friction + sponge + CFL epilogue)")
    roofline = {"bound": "hbm", "kernel": kname,
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6.65 TB/s",
                "traffic": traffic, "algorithmic_bytes_per_launch": st2_bytes,
                "avg_launch_ms": avg["stage2"],
                "step_phase_ms": avg,
                "limiter": "dry tiles: HBM traffic (settled tiles move nothing); wet tiles: FP64 instruction "
                           "issue and dependent-FP64 latency (the all_wet object gives their rate and FP64 pipe "
                           "share)",
                "note": "fraction of HBM over the beach, most of which is dry land that settled tiles skip"}

    # e2e through the C ABI with host buffers: per step upload (h, hu, hv)
    # from pinned host memory, one self-timed step, download (h, hu, hv).
    N = (NX + 4) * (NY + 4)
    pinned = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(3)]
    for q, f in enumerate(("h", "hu", "hv")):
        pinned[q].numpy()[:] = sim.field(f)
    ptrs = [ctypes.cast(p.data_ptr(), ctypes.POINTER(ctypes.c_double)) for p in pinned]
    e2e_steps = max(3, min(K, 40))
    taken = ctypes.c_double()

    def e2e_step():
        for q in range(3):
            swe._lib.check(lib.swe_set_field(sim._h, 1 + q, ptrs[q]))
        swe._lib.check(lib.swe_step_auto(sim._h, ctypes.byref(taken)))
        for q in range(3):
            swe._lib.check(lib.swe_get_field(sim._h, 1 + q, ptrs[q]))

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = world * NX * NY * e2e_steps / float(t.item())

    # device-resident drop-in use: the driver loop sim.step(sim.maxDt())
    # with the state on the device and dt crossing to the host each step
    t0 = time.perf_counter()
    res_steps = max(3, min(K, 200))
    for _ in range(res_steps):
        swe._lib.check(lib.swe_step_auto(sim._h, ctypes.byref(taken)))
    sim.synchronize()
    res_value = NX * NY * res_steps / (time.perf_counter() - t0)

    n_launches = launches_per_step(swe, lib, sim) * K
    lcfg = launch_cfg(swe, lib, sim)
    sim.close()
    cpu = None
    extras = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(b, eta, threads=1)
    if rank == 0 and world == 1 and not args.no_extras:
        # the whole configuration: 2000 steps from the initial state, so the
        # rate covers the flooding of the beach and not only its first steps
        full = make_sim(swe, b, eta)
        full_steps = 2000
        done, ms_full, clocks_full = timed_on(torch, stream_of(swe, full), lambda: full.run(full_steps), local)
        full.close()
        extras["full_run"] = {"steps": full_steps, "done": done, "value": NX * NY * done / (ms_full / 1e3),
                              "unit": UNIT, "ms_per_step": ms_full / full_steps, "clocks": clocks_full,
                              "how": "a fresh simulation of the same workload run through all 2000 steps of "
                                     "the configuration (swe_run), CUDA events on its stream"}
        extras["all_wet"] = all_wet_summary(torch, swe, max(K, 200), local)
        extras["batched"] = ensemble_summary(torch, swe, device=local)
        extras["adjoint"] = adjoint_summary(torch, swe, device=local)
        extras["fma_build"] = fma_build_summary(K, args.warmup)

    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": config({"parallelism": f"independent basin per GPU x{world}",
                                  "launch": dict(zip(["grid_x", "grid_y", "threads", "cols_per_cta",
                                                      "rows_per_cta"], lcfg))}),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8,
                        "d2h_bytes_per_step": 3 * N * 8 + 8,
                        "how": "per step: swe_set_field x3 from pinned host memory, swe_step_auto, "
                               "swe_get_field x3 into pinned host memory"},
                "e2e_resident": {"value": res_value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                 "d2h_bytes_per_step": 8,
                                 "how": "per step: swe_step_auto (dt = maxDt read back), state on the device"},
                "gpu_launches": n_launches,
                "roofline": roofline, "clocks": clocks, "cpu_baseline": cpu,
                "hbm_bytes_per_cell_update": STEP_BYTES}
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def fma_build_summary(steps, warmup):
    """The production build (libswe_b200_fma.so, -fmad=true: the compiler
    fuses multiply-adds; held to 1e-12 per step against the oracle by its
    own test) on the same beach steps and on the all-wet grid, each in a
    child process, since a process loads one build."""
    lib = os.path.join(ROOT, "water-simulator_b200", "libswe_b200_fma.so")
    if not os.path.exists(lib):
        return {"unavailable": "libswe_b200_fma.so is not built"}
    env = dict(os.environ, SWE_B200_ARITH="fma")
    out = {"how": "bench.py in a child process with SWE_B200_ARITH=fma"}
    for key, extra in (("value", ["--no-cpu-baseline", "--no-extras", "--steps", str(steps), "--warmup", str(warmup)]),
                       ("all_wet", ["--workload", "allwet", "--steps", "200", "--warmup", "32"])):
        try:
            r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + extra, env=env,
                               capture_output=True, text=True, timeout=600)
            lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out[key] = json.loads(lines[-1])["value"] if r.returncode == 0 and lines else None
        except (subprocess.TimeoutExpired, ValueError, KeyError) as e:
            out[key] = None
            out[key + "_error"] = str(e)[:200]
    out["unit"] = UNIT
    return out


def launches_per_step(swe, lib, sim):
    """Kernel launches of one step: prepare, two ghost fills and two stages
    of the stage kernels in use (the tiled pair per stage and one close of
    the step, or the fused kernel per stage)."""
    impl = ctypes.c_int(-1)
    swe._lib.check(lib.swe_get_stage_kernels(sim._h, ctypes.byref(impl)))
    # the tiled pair per stage and one close; with tile lists each ghost fill
    # makes the next stage's lists in the same launch
    return 3 + (5 if impl.value == 1 else 2)


def launch_cfg(swe, lib, sim):
    cfg = (ctypes.c_int * 5)()
    swe._lib.check(lib.swe_get_launch_config(sim._h, cfg))
    return list(cfg)


def run_ensemble(args):
    """256 basins of uneven sizes: the batched persistent form against the
    plain single-grid kernel launched per basin (each basin's steps through
    its own device loop), same basins, same number of steps.  Under torchrun
    the basins are spread over the ranks (longest first onto the least
    loaded rank; no collective on the data path), each rank advances its own
    share batched, and the job's time is the slowest rank's (strong scaling:
    the 256 basins are the whole job at every N)."""
    import torch
    import __graft_entry__
    swe = __graft_entry__.load_package()
    from water_simulator_b200 import workloads, sharding
    rank, world, local = sharding.rank_env()
    if world > 1:
        torch.cuda.set_device(local)
        sharding.init_ranks("nccl", device=torch.device("cuda", local))
    swe._lib.check(swe.load_library().swe_set_device(local))
    all_bs = workloads.ensemble()
    total_cells = sum(b["nx"] * b["ny"] for b in all_bs)
    mine = sharding.assign_basins([b["nx"] * b["ny"] for b in all_bs], world)[rank]
    bs = [all_bs[q] for q in mine]
    cells = sum(b["nx"] * b["ny"] for b in bs)
    K = max(4, min(args.steps, 1000))               # the configuration's 1000 steps by default
    ens = swe.Ensemble(bs)
    tuned = ens.autotune(trial_steps=3)
    ens.run(max(args.warmup, 3))
    ens.synchronize()
    st = torch.cuda.ExternalStream(ens.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sharding.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    time.sleep(0.3)
    e0.record(st)
    ens.run(K)
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    ms_batch = sharding.max_over_ranks(e0.elapsed_time(e1), device=torch.device("cuda", local))
    clocks = sampler.stop()
    sharding.barrier()
    batched = total_cells * K / (ms_batch / 1e3)
    ens.close()
    if world > 1:
        if rank == 0:
            print(json.dumps({
                "metric": "FP64 cell-updates/s, batched ensemble", "value": batched, "unit": UNIT, "n_gpus": world,
                "steps": K, "warmup": args.warmup, "ms_per_step": ms_batch / K, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": {"workload": "256 Cartesian basins (see the 1-GPU line), spread over the ranks longest "
                                       "first", "cells": total_cells, "rank0_basins": len(bs),
                           "rank0_cells": cells, "schedule": tuned},
                "gpu_launches": (3 + 2 * (2 if tuned["rows"] == 0 else 1)) * K, "clocks": clocks}))
        torch.distributed.destroy_process_group()
        return 0
    # plain: one ShallowWater per basin, device time of its K steps summed
    lib = swe.load_library()
    ms_plain = 0.0
    for b in bs:
        sim = swe.ShallowWater(nx=b["nx"], ny=b["ny"], dx=b["dx"], bed=b["b"], eta0=b["eta0"], manning=b["manning"])
        t = b["tide"]
        tide = swe.Tide({"X": [t["amp"][0], t["phase_deg"][0]]}, msl=t["msl"],
                        periods_hours={"X": 2 * math.pi / t["omega"][0] / 3600})
        tide.terms[0]["omega"] = t["omega"][0]
        sim.boundaries = {"west": swe.flather(tide.signal())}
        sim.run(max(args.warmup, 3))
        sp = ctypes.c_void_p()
        lib.swe_get_stream(sim._h, ctypes.byref(sp))
        pst = torch.cuda.ExternalStream(sp.value)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(pst)
        sim.run(K)
        a1.record(pst)
        a1.synchronize()
        ms_plain += a0.elapsed_time(a1)
        sim.close()
    plain = cells * K / (ms_plain / 1e3)
    line = {"metric": "FP64 cell-updates/s, batched ensemble", "value": batched, "unit": UNIT, "n_gpus": 1,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms_batch / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "256 Cartesian basins, nx~U[64,1024], ny~U[64,512], dx 5 m, bump+roughness "
                                   "beds, still 2 m, Manning~U[0.015,0.04], west Flather tide 0.5 m, "
                                   "period~U[2,14] h", "cells": cells, "schedule": tuned},
            "plain_per_basin": {"value": plain, "unit": UNIT, "ms_per_step": ms_plain / K,
                                "how": "swe_run per basin, device time summed"},
            "batched_over_plain": batched / plain,
            "gpu_launches": (3 + 2 * (2 if tuned["rows"] == 0 else 1)) * K, "clocks": clocks}
    print(json.dumps(line))
    return 0


def run_slabs(args):
    """One 2048 x 2048 beach cut into row slabs over the ranks (strong
    scaling: the grid is the whole job at every N).  Each rank steps its slab
    on its own GPU; halos (6 rows of h, hu, hv each side) move between
    neighbours by NCCL point-to-point from device buffers, and dt is the
    all-reduce MIN of the slabs' maxDt() on the device -- no host round trip
    per step.  With one rank the single slab is the grid."""
    import torch
    import __graft_entry__
    swe = __graft_entry__.load_package()
    from water_simulator_b200 import slabs, sharding
    from water_simulator_b200.workloads import beach_dam_break
    rank, world, local = sharding.rank_env()
    torch.cuda.set_device(local)
    if world > 1:
        sharding.init_ranks("nccl", device=torch.device("cuda", local))
    swe._lib.check(swe.load_library().swe_set_device(local))
    b, h = beach_dam_break(NX, NY, DX)
    eta = b + h
    a, c = slabs.slab_rows(NY, world)[rank]
    slab = slabs.Slab(NY, a, c)
    sim = swe.ShallowWater(nx=NX, ny=slab.rows, dx=DX, bed=slab.take(b), eta0=slab.take(eta), manning=MANNING)
    sim.boundaries = {"west": swe.flather(swe.Tide({}, msl=0.0).signal()), "east": swe.reflect,
                      "south": swe.reflect, "north": swe.reflect}
    sim._prepare_flather()
    if world > 1:
        run = slabs.DistributedSlab(slab, sim, torch.distributed, device=f"cuda:{local}")
    else:
        run = slabs.LocalSlabs([slab], [sim], device=True)
    for _ in range(max(args.warmup, 3)):
        run.step()
    torch.cuda.synchronize()
    K = args.steps
    sharding.barrier()
    st = torch.cuda.ExternalStream(stream_of(swe, sim))
    sampler = ClockSampler(local)
    time.sleep(0.25)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(K):
        run.step()
    e1.record(st)
    torch.cuda.synchronize()
    ms = sharding.max_over_ranks(e0.elapsed_time(e1), device=torch.device("cuda", local))
    clocks = sampler.stop()
    sharding.barrier()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": NX * NY * K / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config({"parallelism": f"row slabs x{world}: 6-row halos by NCCL point-to-point from "
                                             "device buffers, dt by a device all-reduce MIN",
                              "rank0_rows": [a, c]}),
            "gpu_launches": None, "clocks": clocks}))
    sim.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


SPHERE_OMEGA = 7.2921e-5
M2_HOURS = 12.42


def run_sphere(args):
    """The 1440 x 720 spherical tide workload (0.25 degrees in longitude,
    band 85S..85N), longitude periodic, Flather M2 tide (1 m, 12.42 h) on
    the south and north cap edges, Coriolis on (Earth's rotation), wetting
    and drying over 30% land, dt = maxDt() each step; 5000 steps through the
    device loop.
    The first steps are checked bit for bit against the oracle on the same
    input, and the oracle gives the CPU baseline on a bounded sample."""
    import torch
    import __graft_entry__
    swe = __graft_entry__.load_package()
    from water_simulator_b200 import workloads
    c = workloads.globe_tide()
    nx, ny = c["nx"], c["ny"]
    sphere = {"R": 6371e3, "lat0": c["lat0"], "lat1": c["lat1"], "omega": SPHERE_OMEGA}
    tide = swe.Tide({"M2": [1.0, 0.0]}, periods_hours={"M2": M2_HOURS})
    K = int(os.environ.get("SWE_SPHERE_STEPS", "5000"))

    def make():
        sim = swe.ShallowWater(nx=nx, ny=ny, bed=c["b"], eta0=c["eta0"], sphere=sphere)
        sim.boundaries = {"south": swe.flather(tide.signal()), "north": swe.flather(tide.signal())}
        return sim

    def oracle(threads):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_sim import OracleSim
        o = OracleSim(nx=nx, ny=ny, bed=c["b"], eta0=c["eta0"], sphere=sphere, threads=threads)
        tr = tide.terms
        row = ("tide", tide.msl, [k["amp"] for k in tr], [k["omega"] for k in tr], [k["phase"] for k in tr], 0.0)
        o.set_boundaries(west="periodic", east="periodic", south=row, north=row)
        return o

    # parity of the first steps at full size (bit-exact fields, same t)
    chk = 3
    sim = make()
    sim.run(chk)
    ref = oracle(os.cpu_count() or 1)
    for _ in range(chk):
        ref.step()
    exact = all(np.array_equal(sim.field(f), ref.field(f)) for f in ("h", "hu", "hv")) and sim.t == ref.t
    rel = max(float(np.max(np.abs(sim.field(f) - ref.field(f))) / max(np.max(np.abs(ref.field(f))), 1e-300))
              for f in ("h", "hu", "hv"))
    ref.close()
    sim.close()

    sim = make()
    sp = ctypes.c_void_p()
    lib = swe.load_library()
    swe._lib.check(lib.swe_get_stream(sim._h, ctypes.byref(sp)))
    st = torch.cuda.ExternalStream(sp.value)
    sim.run(max(args.warmup, 3))
    sim.synchronize()
    sampler = ClockSampler(0)
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    done = sim.run(K)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    if done != K:
        raise RuntimeError(f"the device loop took {done} of {K} steps")
    value = nx * ny * K / (ms / 1e3)
    dt_last = sim.maxDt()
    finite = sim.finite()
    per_step = launches_per_step(swe, lib, sim)
    sim.close()
    cpu = None
    if not args.no_cpu_baseline:
        o = oracle(1)
        o.step()
        n, t0 = 0, time.perf_counter()
        while True:
            o.step()
            n += 1
            el = time.perf_counter() - t0
            if el >= 12.0 or n >= 40:
                break
        o.close()
        cpu = {"value": nx * ny * n / el, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{n} self-timed steps of the same sphere workload ({el:.1f} s) on the oracle, 1 thread"}
    line = {"metric": "FP64 cell-updates/s, sphere", "value": value, "unit": UNIT, "n_gpus": 1, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"sphere {nx}x{ny}, 0.25 deg longitude, lat {c['lat0']}..{c['lat1']} "
                                   "(the whole sphere has no open edge), band-limited bed 0-5000 m deep with the "
                                   "30% highest cells land at +50 m, still water, Flather M2 tide 1 m (12.42 h) on "
                                   "the S and N cap edges, Coriolis omega 7.2921e-5, Manning 0.025, dt = maxDt()",
                       "cells": nx * ny, "l2": "state 3 x 8.4 MB per copy: fits L2; steady-state stream"},
            "first_steps_vs_oracle": {"steps": chk, "bit_exact": exact, "max_rel_err": rel}, "finite": finite, "dt_last": dt_last,
            "gpu_launches": per_step * K, "clocks": clocks, "cpu_baseline": cpu}
    print(json.dumps(line))
    return 0


def run_adjoint(args):
    """Gradient of the gauge misfit on the 1024 x 1024 case: the cost of one
    gradient (forward with checkpoints + backward) against the plain forward
    of the same steps, and a central-difference check on random directions."""
    import torch
    import __graft_entry__
    swe = __graft_entry__.load_package()
    from water_simulator_b200 import workloads
    n = int(os.environ.get("SWE_ADJ_N", "1024"))
    steps = int(os.environ.get("SWE_ADJ_STEPS", "2000"))
    ndir = int(os.environ.get("SWE_ADJ_DIRS", "20"))
    c = workloads.adjoint_case(nx=n, ny=n, dx=10.0, n_gauges=32)
    kw = dict(manning_field=c["n"], gauges=c["gauges"], steps=steps, checkpoint_every=45)
    truth = swe.MisfitAdjoint(n, n, 10.0, c["b_true"], c["eta0"], **kw)
    _, obs = truth.forward()
    truth.close()
    def timed(stream_ptr, fn):
        st = torch.cuda.ExternalStream(stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        out = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    def stream_of(sim):
        sp = ctypes.c_void_p()
        swe._lib.check(swe._lib.load().swe_get_stream(sim._h, ctypes.byref(sp)))
        return sp.value

    # plain forward: the same self-timed steps through the device loop (warm one run first)
    t_plain = None
    for _ in range(2):
        sim = swe.ShallowWater(nx=n, ny=n, dx=10.0, bed=c["b"], eta0=c["eta0"])
        sim.setManningField(c["n"])
        sim.synchronize()
        _, t_plain = timed(stream_of(sim), lambda: sim.run(steps))
        sim.close()
    adj = swe.MisfitAdjoint(n, n, 10.0, c["b"], c["eta0"], **kw)
    adj.set_observations(obs)
    adj.forward()                     # warm-up gradient: the tape is allocated on the first backward
    adj.backward()
    (J, _), t_fwd = timed(adj.stream(), adj.forward)
    (gb, gn), t_bwd = timed(adj.stream(), adj.backward)
    dts = adj.dt_sequence()
    rng = np.random.default_rng(7)
    errs = []
    for _ in range(ndir):
        db = rng.normal(0, 1, c["b"].shape)
        dn = rng.normal(0, 1e-3, c["n"].shape)
        want = float(np.dot(gb, db.reshape(-1)) + np.dot(gn, dn.reshape(-1)))
        best = math.inf
        for eps in (1e-6, 1e-5, 1e-7):
            vals = []
            for sgn in (1, -1):
                f = swe.MisfitAdjoint(n, n, 10.0, c["b"] + sgn * eps * db, c["eta0"],
                                      **dict(kw, manning_field=c["n"] + sgn * eps * dn, checkpoint_every=steps))
                f.set_observations(obs)
                f.dt_sequence(fixed=dts)
                vals.append(f.forward()[0])
                f.close()
            best = min(best, abs((vals[0] - vals[1]) / (2 * eps) - want) / abs(want))
            if best <= 1e-5:
                break
        errs.append(best)
    adj.close()
    line = {"metric": "adjoint gradient / forward time ratio", "value": (t_fwd + t_bwd) / t_plain,
            "unit": "x forward", "higher_is_better": False, "n_gpus": 1, "steps": steps, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{n}x{n} dx=10 m, bump+roughness bed, 0.5 m released hump over 2 m still water, "
                                   "Manning field U[0.015,0.04], 32 gauges, observations from bed + N(0,0.1) noise, "
                                   "checkpoint every 45 steps", "cells": n * n},
            "forward_plain_s": t_plain, "forward_recording_s": t_fwd, "backward_s": t_bwd,
            "backward_over_forward": t_bwd / t_plain, "J": J,
            "fd_check": {"directions": ndir, "max_rel_err": max(errs) if errs else None,
                         "median_rel_err": float(np.median(errs)) if errs else None}}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.stage != "default":
        os.environ["SWE_B200_STAGE"] = args.stage
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        return run_ensemble(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "sphere":
        return run_sphere(args)
    if args.workload == "slabs":
        return run_slabs(args)
    if args.workload == "allwet":
        import torch
        import __graft_entry__
        swe = __graft_entry__.load_package()
        line = all_wet_summary(torch, swe, args.steps, 0, warm=max(args.warmup, 3))
        line.update(metric="FP64 cell-updates/s, all-wet 2048x2048", n_gpus=1, warmup=args.warmup,
                    higher_is_better=True, dtype="f64", data="synthetic (seeded)")
        print(json.dumps(line))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
