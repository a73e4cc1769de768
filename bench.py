"""Benchmark of the fused monodomain step: cell-steps/s on the 256^3 box
(BetterTT06 + FGR 19-point stencil + face pacing, dt = 0.02 ms), mixed
FP32/FP64 (headline) and FP64, one fused kernel per time step.

    python bench.py [--gpus N --steps K --warmup W]       # our engine
    python bench.py --impl reference [...]                 # the reference CPU path

One process per GPU (torchrun for N > 1); each GPU runs its own 256^3 tissue
(independent tissues shard with no data-path collective: weak scaling).
Prints one JSON line on rank 0.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 0.02
METRIC = "cell-steps/s"
# algorithmic bytes per cell-step of one fused step (compulsory HBM traffic):
# Vm read+write 16 B; state FP64 18x8x2 = 288 B, mixed 5x8x2 + 13x4x2 = 184 B;
# stencil weights FP64 19x8 = 152 B, mixed 18x4 = 72 B; the cell's voxel
# offset 4 B (the reaction type is per warp tile, not per cell).
ALGO_BYTES = {"fp64": 16 + 288 + 152 + 4, "mixed": 16 + 184 + 72 + 4}


def workload(name):
    if name == "box256":
        return dict(nx=256, ny=256, nz=256, period=500.0, label="box256: 256^3 = 16,777,216 cells, dx 0.2 mm, "
                    "endo/mid/epi x-slabs 25/35/40 %, fibre -60..+60 deg across z, sigma_l 0.133 / sigma_t 0.0176 S/m, "
                    "beta 1400/cm, Cm 1 uF/cm^2, S1 pacing every 500 ms on the x = 0 face, dt 0.02 ms")
    if name == "box192":
        return dict(nx=192, ny=192, nz=192, period=500.0, label="box192: 192^3 = 7,077,888 cells (traffic capture "
                    "size: every launch writes far more than L2), otherwise as box256")
    if name == "box128":
        return dict(nx=128, ny=128, nz=128, period=500.0, label="box128: 128^3 = 2,097,152 cells (profiling size), "
                    "otherwise as box256")
    if name == "box64":
        return dict(nx=64, ny=64, nz=64, period=1000.0, label="box64: 64^3 = 262,144 cells, single stimulus at t = 0 "
                    "on the x = 0 face, otherwise as box256")
    raise ValueError(name)


def bench_config(w, world):
    """The `config` object of both arms' lines (same workload, same keys)."""
    n = w["nx"] * w["ny"] * w["nz"]
    return {"workload": w["label"], "cells_per_gpu": n, "dt_ms": DT,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (state + weights %.1f GB per GPU, mixed)" % (
                (ALGO_BYTES["mixed"] - 16) * n / 1e9)}


def tuning_overrides(e, stage=None, ctas=None, layout=None):
    """Profiling runs: forces the staging mode, the CTAs per SM and the tile
    layout where given (before any tissue is added)."""
    if layout is not None:
        e.set_layout(layout)
    if stage is not None or ctas is not None:
        st, ct = e.get_tuning()
        e.set_tuning(st if stage is None else stage, ct if ctas is None else ctas)


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s)"


def read_traffic(precision):
    """DRAM bytes per cell-step of the fused kernel from the committed ncu
    summary (profiles/fused_step_traffic.json), if one exists."""
    path = os.path.join(ROOT, "profiles", "fused_step_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    v = d.get(precision, {}).get("dram_bytes_per_cell_step")
    return float(v) if v is not None else None


# ---------------------------------------------------------------- CPU side

def _cpu_worker(args):
    """Runs the reference CPU path (oracle/_ref) or the oracle port on the
    workload's box, or on one z-slab of it, with `threads` OpenMP threads
    (the reference's omp loop: the FGR stencil threaded, BetterTT06
    single-threaded); returns (cells, steps, seconds, set-up seconds)."""
    kind, box, zrange, steps, warmup, threads = args
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cardioid_b200 import engine, tissue
    s0 = time.perf_counter()
    t = tissue.box(box["nx"], box["ny"], box["nz"], period=box["period"], seed=1234, zrange=zrange)
    if kind == "reference":
        from golden.make_golden import reference_sim
        from oracle import refsim
        refsim.set_threads(threads)
        sim = reference_sim(t)
        sim.set_vm(t.vm0)
    else:
        from oracle import port
        params = [engine.default_params(ct, DT) for ct in (0, 1, 2)]
        sim = port.PortSim(t, params, (t.cell_type - 100).astype(np.uint8), DT)
    setup = time.perf_counter() - s0
    sim.step(warmup)
    t0 = time.perf_counter()
    sim.step(steps)
    return t.n, steps, time.perf_counter() - t0, setup


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return ""


def cpu_baseline(box, steps, warmup, omp_steps=2, procs=None):
    """The reference's CPU path on the workload's own geometry.

    value: one single-threaded process per host core, each stepping one
    z-slab of the box (the decomposition the reference gives its MPI ranks,
    here without the halo exchange: slab faces are no-flux), `steps` steps
    after `warmup`; the rate is all cells x steps / the slowest process.
    omp_loop_one_process: the whole box in one process, the reference's omp
    loop as shipped (stencil on every core, reaction on one), `omp_steps`
    steps after one warm-up step."""
    from oracle import refsim
    kind = "reference" if refsim.available() else "port"
    procs = procs or os.cpu_count() or 1
    nz = box["nz"]
    cuts = [round(nz * r / procs) for r in range(procs + 1)]
    jobs = [(kind, box, (cuts[r], cuts[r + 1]), steps, warmup, 1) for r in range(procs) if cuts[r + 1] > cuts[r]]
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(_cpu_worker, jobs)
    cells = sum(r[0] for r in res)
    wall = max(r[2] for r in res)
    per_core = sum(r[0] * r[1] / r[2] for r in res) / len(res)
    out = {"value": cells * steps / wall, "unit": METRIC, "cores": procs, "kind": kind, "per_core": per_core,
           "cells": cells, "steps": steps}
    what = ("the reference's own CPU path (oracle/_ref: BetterTT06 via ReactionManager + FGRDiffusionOMP + "
            "BoxStimulus, omp-loop order)" if kind == "reference" else "the oracle's C restatement of the reference path")
    omp = None
    if omp_steps > 0:
        with ctx.Pool(1) as pool:
            n1, s1, w1, su1 = pool.map(_cpu_worker, [(kind, box, None, omp_steps, 1, procs)])[0]
        omp = n1 * s1 / w1
        out["omp_loop_one_process"] = omp
        out["omp_loop_setup_s"] = su1
    out["sample"] = (
        "%s on the %dx%dx%d box (%d cells): %d processes, one per host core, each a z-slab of the box (the "
        "reference's MPI-style decomposition, no halo exchange), %d steps after %d warm-up; omp_loop_one_process: "
        "the whole box in one process, stencil on %d OpenMP threads and the reaction on one as the reference's omp "
        "loop runs, %d steps after 1 warm-up; CPU: %s" % (what, box["nx"], box["ny"], nz, cells, len(jobs), steps,
                                                          warmup, procs, omp_steps, _cpu_model()))
    return out


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock and clock-event reasons of one GPU during a timed region.

    The caller polls: `sample()` reads the current SM clock and the active
    clock-event reasons through NVML (well under a millisecond per call), so
    a timed region of a few milliseconds still gets samples.  Without NVML
    it falls back to `nvidia-smi -lms 200` in the background (long regions
    only)."""
    NVML_REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                    ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.nvml = None
        self.sm, self.reasons, self.max_mhz = [], set(), None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        return pynvml, h

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            pynvml, h = self.nvml
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.sample()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def sample(self):
        if not self.nvml:
            return
        pynvml, h = self.nvml
        try:
            self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
            bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            return
        for name, bit in self.NVML_REASONS:
            if bits & bit:
                self.reasons.add(name)

    def wait(self, event, every_s=0.002):
        """Samples every `every_s` seconds until the CUDA event has completed."""
        self.sample()
        while not event.query():
            self.sample()
            time.sleep(every_s)
        self.sample()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml:
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if self.nvml:
            if not self.sm:
                return None
            return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "NVML, polled every 2 ms"}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi -lms 200"}


# ---------------------------------------------------------------- GPU side

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            # processes without a GPU (the CPU test of this plumbing): gloo
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, local):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda:%d" % local if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def batch_of(steps, most=50):
    """The launch-batch length the timed steps run in: the largest divisor of
    steps not above `most`, so one CUDA graph (captured during warm-up)
    replays through the whole timed region."""
    return max(d for d in range(1, min(steps, most) + 1) if steps % d == 0)


def time_engine(e, steps, warmup, world, local):
    import torch
    stream = torch.cuda.ExternalStream(e.stream(), device="cuda:%d" % local)
    k = batch_of(steps)
    e.step(warmup)
    e.step(k)            # untimed: captures the graph the timed region replays
    e.sync()
    torch.cuda.synchronize(local)
    barrier(world)
    l0 = e.launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(steps // k):
            e.step(k)
        stop.record(stream)
        clk.wait(stop)
        stop.synchronize()
    torch.cuda.synchronize(local)
    ms = start.elapsed_time(stop)
    barrier(world)
    return ms, e.launch_count() - l0, clk.summary()


def run_ours(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from cardioid_b200 import engine, tissue
    w = workload(args.config)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, args.cpu_steps, 2, args.cpu_omp_steps)   # before the first GPU call
    t = tissue.box(w["nx"], w["ny"], w["nz"], period=w["period"], seed=1234 + rank)
    n = t.n
    peak, peak_src = read_peaks()
    results = {}
    precs = ("fp64", "mixed") if args.precision == "both" else (args.precision,)
    finals = {}
    from cardioid_b200 import autotune
    for prec in precs:
        choice = None
        if not args.no_autotune and args.stage is None and args.ctas is None and args.layout is None:
            # tile layout and staging timed on this box (same bits for every choice)
            choice = autotune.tune(lambda: engine.Engine(DT, precision=prec, device=local),
                                   lambda e: e.add_tissue(t, engine.transmural_setup(e, t, DT)[0]),
                                   w["label"].split(":")[0], steps=20, stage_modes=(0, 2, 3), ctas_per_sm=(0,))
        with engine.Engine(DT, precision=prec, device=local) as e:
            if choice:
                autotune.apply(e, choice)
            tuning_overrides(e, args.stage, args.ctas, args.layout)
            rx, _ = engine.transmural_setup(e, t, DT)
            e.add_tissue(t, rx)
            ms, launches, clocks = time_engine(e, args.steps, args.warmup, world, local)
            ms = max_over_ranks(ms, world, local)
            finals[prec] = (e.read_vm(0), e.read_activation(0), e.time(0)[0])
            per_launch_s = ms / 1e3 / args.steps
            achieved = ALGO_BYTES[prec] * n / per_launch_s / 1e9
            traffic_pc = read_traffic(prec)
            results[prec] = {
                "value": world * n * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                "tuning": {"layout": e.get_layout(), "stage": e.get_tuning()[0], "ctas_per_sm": e.get_tuning()[1],
                           "autotune_table_ms_per_step": choice["table"] if choice else None},
                "gpu_launches": launches, "clocks": clocks,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": peak_src,
                             "algorithmic_bytes_per_cell_step": ALGO_BYTES[prec],
                             "traffic": (traffic_pc * n if traffic_pc else None)},
            }
            if prec == "mixed" and not args.no_e2e:
                # end to end through the C ABI with host buffers: every step
                # copies Vm in from pinned host memory and the new Vm back
                vin = torch.from_numpy(t.vm0.copy()).pin_memory()
                vout = torch.empty_like(vin).pin_memory()
                vin_np, vout_np = vin.numpy(), vout.numpy()
                e2e_steps = max(1, min(args.steps, args.e2e_steps))
                for _ in range(args.warmup):
                    e.step_host(0, vin_np, vout_np)
                barrier(world)
                t0 = time.perf_counter()
                for _ in range(e2e_steps):
                    e.step_host(0, vin_np, vout_np)
                    vin_np, vout_np = vout_np, vin_np
                el = max_over_ranks(time.perf_counter() - t0, world, local)
                results["e2e"] = {"value": world * n * e2e_steps / el, "unit": METRIC,
                                  "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                                  "steps": e2e_steps,
                                  "call": "cdb_engine_step_host (pinned host Vm in, one fused step, host Vm out)"}
    if rank != 0:
        return
    if args.precision != "both" or args.no_e2e:
        # a profiling run: one line per precision, no headline
        for prec in precs:
            extra = {"e2e": results["e2e"]} if prec == "mixed" and "e2e" in results else {}
            print(json.dumps({"config": w["label"], "precision": prec, "steps": args.steps, **results[prec], **extra}),
                  flush=True)
        return
    m, f = results["mixed"], results["fp64"]
    (vf, af, sf), (vm_, am, sm_) = finals["fp64"], finals["mixed"]
    both = (af > 0) & (am > 0)
    errors = {"steps": int(sf), "max_abs_dvm_mV": float(np.abs(vm_ - vf).max()),
              "activated_fp64": int((af > 0).sum()), "activated_mixed": int((am > 0).sum()),
              "activation_max_err_ms": float(np.abs(af[both] - am[both]).max()) if both.any() else None,
              "full_beat": apd_check(local) if world == 1 and not args.no_apd else None}
    plain = time_plain_fp64(t, args, local) if world == 1 and not args.no_plain else None
    ref_gpu = reference_gpu_block(t, local) if world == 1 and not args.no_plain else None
    ref_gpu_diff = reference_gpu_diffusion_block(local) if world == 1 and not args.no_plain else None
    # configs 2 and 4 in the same line (one GPU only, to keep the run short)
    shell_line = shell_block(args.shell_steps, args.shell_dx, world, rank, local) \
        if world == 1 and not args.no_shell else None
    serve_line = serve_block(args.line_jobs, args.rate, args.job_steps, args.job_beats, ("mixed",), args.serve_batch,
                             world, rank, local) if world == 1 and not args.no_serve else None
    line = {
        "metric": METRIC, "value": m["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (mixed: FP32 fits/gates/currents/stencil, FP64 Vm and concentrations)",
        "data": "synthetic, seeded (no dataset: the configs define geometry, fibres and pacing)",
        "config": bench_config(w, world),
        "precision": "mixed",
        "timing": "one CUDA graph of %d steps, captured during warm-up, replayed %d times" % (
            batch_of(args.steps), args.steps // batch_of(args.steps)),
        "impl": "ours",
        "roofline": m["roofline"],
        "tuning": m["tuning"],
        "fp64": {"value": f["value"], "ms_per_step": f["ms_per_step"], "roofline": f["roofline"],
                 "dtype": "f64", "tuning": f["tuning"]},
        "mixed_over_fp64": m["value"] / f["value"],
        "mixed_vs_fp64": errors,
        "plain_fp64": plain,
        "mixed_over_plain_fp64": (m["value"] / plain["value"]) if plain else None,
        "reference_gpu_reaction": ref_gpu,
        "reference_gpu_diffusion": ref_gpu_diff,
        "e2e": results["e2e"],
        "shell": shell_line,
        "serve": serve_line,
        "gpu_launches": m["gpu_launches"],
        "clocks": m["clocks"],
        "clocks_fp64": f["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def _timed_run(e, steps, warmup, world, local):
    ms, launches, clocks = time_engine(e, steps, warmup, world, local)
    return max_over_ranks(ms, world, local), launches, clocks


def shell_block(steps, dx, world, rank, local, warmup=3, overrides=None):
    """Irregular anatomy (config 2): the truncated prolate-ellipsoid shell at
    dx mm (20 paced endocardial sites), FP64 and mixed, each timed over
    `steps` steps after `warmup`, and the mixed path's activation-time error
    against FP64 over those steps."""
    from cardioid_b200 import engine, shell
    t = shell.prolate_shell(dx=dx, seed=1234 + rank)
    rx = (t.cell_type - 100).astype(np.uint8)
    out, acts = {}, {}
    for prec in ("fp64", "mixed"):
        with engine.Engine(DT, precision=prec, device=local) as e:
            tuning_overrides(e, **(overrides or {}))
            rid = [e.add_reaction(engine.default_params(c, DT)) for c in (0, 1, 2)]
            tid = e.add_tissue(t, np.array(rid, np.uint8)[rx])
            ms, launches, clocks = _timed_run(e, steps, warmup, world, local)
            acts[prec] = e.read_activation(tid)
            out[prec] = {"value": world * t.n * steps / (ms / 1e3), "ms_per_step": ms / steps,
                         "gpu_launches": launches, "clocks": clocks}
    a, b = acts["fp64"], acts["mixed"]
    both = (a > 0) & (b > 0)
    return {"metric": METRIC, "unit": METRIC,
            "workload": "prolate shell %.3g mm (config 2): %d cells on a %dx%dx%d grid, 64-bit voxel indices, "
                        "20 paced endocardial sites, %d steps (+%d warm-up) at dt %g"
                        % (dx, t.n, t.nx, t.ny, t.nz, steps, warmup, DT),
            "n_gpus": world, "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "mixed_vs_fp64": {"activated_fp64": int((a > 0).sum()), "activated_mixed": int((b > 0).sum()),
                              "activation_max_err_ms": float(np.abs(a[both] - b[both]).max()) if both.any() else None}}


def overrides_of(args):
    return {"stage": args.stage, "ctas": args.ctas, "layout": args.layout}


def run_shell(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    line = shell_block(args.steps, args.shell_dx, world, rank, local, overrides=overrides_of(args))
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch(args):
    """Many instances in one engine: a seeded population (4096 cables,
    sheets and boxes, per-instance cell type, conductance scales and cycle
    length); sustained cell-steps/s over the timed steps."""
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from cardioid_b200 import engine, population as pop
    from cardioid_b200 import autotune
    insts = pop.draw(pop.PopulationSpec(n=args.instances), seed=1234)
    mine = [i for i in insts if i.index % world == rank]
    out = {}
    for prec in args.batch_precisions.split(","):
        choice = None
        if not args.no_autotune:
            # tile layout, staging and grid chosen on a sample of the population
            sample = mine[::max(1, len(mine) // 96)]

            def make():
                e = engine.Engine(DT, precision=prec, device=local)
                for c in (0, 1, 2):
                    e.add_reaction(engine.default_params(c, DT))
                return e

            def add(e):
                for inst in sample:
                    t = pop.build(inst)
                    e.add_tissue(t, np.full(t.n, inst.celltype, np.uint8), scales=inst.scales)

            choice = autotune.tune(make, add, "population-%d" % args.instances)
        with engine.Engine(DT, precision=prec, device=local) as e:
            rid = [e.add_reaction(engine.default_params(c, DT)) for c in (0, 1, 2)]
            if choice:
                autotune.apply(e, choice)
            t0 = time.perf_counter()
            for inst in mine:
                t = pop.build(inst)
                e.add_tissue(t, np.full(t.n, rid[inst.celltype], np.uint8), scales=inst.scales)
            setup = time.perf_counter() - t0
            ms, launches, clocks = _timed_run(e, args.steps, 3, world, local)
            # every rank steps its share; the time is the slowest rank's
            out[prec] = {"value": pop.total_cells(insts) * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                         "gpu_launches": launches, "setup_s": setup, "clocks": clocks,
                         "tuning": {"layout": e.get_layout(), "stage": e.get_tuning()[0],
                                    "ctas_per_sm": e.get_tuning()[1],
                                    "autotune_table_ms_per_step": choice["table"] if choice else None}}
    if rank == 0:
        print(json.dumps({"metric": METRIC, "unit": METRIC, "n_gpus": world,
                          "workload": "population of %d instances (%d cells), steps %d (+3 warm-up) at dt %g"
                          % (len(insts), pop.total_cells(insts), args.steps, DT), **out}), flush=True)


def serve_block(n_jobs, rate, job_steps, job_beats, precisions, serve_batch, world, rank, local, overrides=None):
    """Serving (config 4): Poisson job arrivals with config 4's size and
    parameter distributions, continuous batching in one engine per
    precision; p50/p99 time-to-result and aggregate cell-steps/s.  Each job
    runs `job_beats` paced beats, or `job_steps` steps when that is given
    (a shortened job, labelled so)."""
    from cardioid_b200 import engine, serving
    spec = serving.JobSpec(rate=rate, steps=job_steps or None, beats=job_beats)
    jobs = serving.partition(serving.draw_jobs(n_jobs, spec, seed=1234), rank, world)
    out = {}
    for prec in precisions:
        with engine.Engine(DT, precision=prec, device=local) as e:
            tuning_overrides(e, **(overrides or {}))
            rid = [e.add_reaction(engine.default_params(c, DT)) for c in (0, 1, 2)]
            srv = serving.Server(e, rid, batch=serve_batch)
            res = srv.run(jobs)
            out[prec] = serving.summary(res, srv.elapsed, srv.cell_steps)
            out[prec]["rejected"] = len(srv.rejected)
    length = ("%d steps (%g ms of simulated time, shortened from config 4's %d paced beats)"
              % (job_steps, job_steps * DT, job_beats) if job_steps else "%d paced beats" % job_beats)
    return {"metric": "time-to-result p50/p99 (s), cell-steps/s", "n_gpus": world,
            "workload": "serving (config 4): %d jobs, Poisson %.3g/s, log-normal sizes (median 2e5, max 3e7 cells), "
                        "each %s at dt %g" % (n_jobs, rate, length, DT), **out}


def run_serve(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    line = serve_block(args.jobs, args.rate, args.job_steps, args.job_beats, tuple(args.serve_precisions.split(",")),
                       args.serve_batch, world, rank, local, overrides=overrides_of(args))
    if rank == 0:
        print(json.dumps(line), flush=True)


def apd_check(local, n=32, steps=20000, every=10, probes=64):
    """Mixed against FP64 over one full paced beat (400 ms) of an n^3 box:
    Vm sampled every `every` steps at `probes` cells spread over the box,
    APD90 per probe (cardioid_b200.sensors.apd90), activation times of every
    cell; the largest differences."""
    from cardioid_b200 import engine, sensors, tissue
    t = tissue.box(n, n, n, period=1000.0, seed=99)
    idx = np.linspace(0, t.n - 1, probes).astype(np.int64)
    tr, act = {}, {}
    times = DT * every * np.arange(1, steps // every + 1)
    for prec in ("fp64", "mixed"):
        with engine.Engine(DT, precision=prec, device=local) as e:
            rx, _ = engine.transmural_setup(e, t, DT)
            tid = e.add_tissue(t, rx)
            rows = []
            for _ in range(steps // every):
                e.step(every)
                rows.append(e.read_vm(tid)[idx])
            tr[prec], act[prec] = np.array(rows), e.read_activation(tid)
    errs, apds = [], []
    for j in range(probes):
        a64, am = sensors.apd90(tr["fp64"][:, j], times), sensors.apd90(tr["mixed"][:, j], times)
        if len(a64) and len(a64) == len(am):
            errs.append(float(np.abs(a64 - am).max()))
            apds.append(float(a64.mean()))
    both = (act["fp64"] > 0) & (act["mixed"] > 0)
    return {"workload": "%d^3 box, one paced beat (%d steps, %g ms), Vm sampled every %d steps at %d probe cells"
                        % (n, steps, steps * DT, every, probes),
            "apd90_probes": len(errs), "apd90_max_err_ms": max(errs) if errs else None,
            "apd90_mean_fp64_ms": float(np.mean(apds)) if apds else None,
            "activation_max_err_ms": float(np.abs(act["fp64"] - act["mixed"])[both].max()) if both.any() else None,
            "activated_fp64": int((act["fp64"] > 0).sum()), "activated_mixed": int((act["mixed"] > 0).sum())}


def time_plain_fp64(t, args, local):
    """The plain FP64 GPU path: the reference's split loop on the drop-in
    plugins (elec/simulationLoop.cc:183-231), one Reaction::calc per
    reaction type (cdb_reaction_calc), Diffusion::updateLocalVoltage and
    calc (cdb_fgr_*), then iStim and Vm += dt (dVmR + dVmD + iStim) as
    tensor operations; Vm crosses HBM several times per step."""
    import torch
    from cardioid_b200 import engine, plugins
    dev = "cuda:%d" % local
    params = [engine.default_params(c, DT) for c in (0, 1, 2)]
    ct = torch.from_numpy(np.asarray(t.cell_type) - 100).to(dev)
    idx = [torch.nonzero(ct == c).flatten().to(torch.int32) for c in (0, 1, 2)]
    rx = [plugins.BetterTT06(params[c], idx[c].numel(), DT) for c in (0, 1, 2)]
    fgr = plugins.FGRDiffusion(t)
    vm = torch.from_numpy(t.vm0.copy()).to(dev)
    dvr, dvd, ist = torch.zeros_like(vm), torch.zeros_like(vm), torch.zeros_like(vm)
    x = torch.from_numpy(np.asarray(t.tuples()[0])).to(dev)
    face = (x > t.stimuli[0].xMin) & (x < t.stimuli[0].xMax)
    amp = t.stimuli[0].amplitude

    def step(n):
        for _ in range(n):
            ist.zero_()
            ist.masked_fill_(face, amp)          # on at t < 1 ms of the first beat only; the cost is the same
            for c in (0, 1, 2):
                rx[c].calc(DT, idx[c], vm, ist, dvr)
            fgr.updateLocalVoltage(vm)
            fgr.calc(dvd)
            vm.add_(DT * (dvr + dvd + ist))
    steps = min(args.steps, 200)
    step(args.warmup)
    torch.cuda.synchronize(local)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    step(steps)
    s1.record()
    s1.synchronize()
    ms = s0.elapsed_time(s1)
    return {"value": t.n * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps, "dtype": "f64",
            "path": "split loop on the plugins: 3 x cdb_reaction_calc + cdb_fgr_update_local_voltage + cdb_fgr_calc "
                    "+ stimulus and Vm update as tensor ops (CUDA events, default stream)"}


def reference_gpu_block(t, local, steps=20, warmup=3):
    """The reference's own GPU reaction (BetterTT06's NVRTC kernel through its
    ReactionManager::calc, oracle/_ref/ref_gpu_reaction, in a child process)
    beside the plugin reaction (plugins.ReactionManager over
    cdb_reaction_calc) on the box's cells: FP64, Vm and iStim fixed at the
    resting state, `steps` calls after `warmup`, CUDA events on each side's
    launching stream.  The reference's GPU diffusion (CUDADiffusion) has
    another stencil rule (6 faces, not FGR's 19 points) and runs only on y
    and z extents that are multiples of 30, so it is timed apart
    (reference_gpu_diffusion_block)."""
    from oracle import refgpu
    if not refgpu.available():
        return None
    import torch
    from cardioid_b200 import engine, objectdb, plugins, tissue
    info, _, _ = refgpu.run(t.cell_type, DT, steps, warmup)
    db = objectdb.ObjectDB()
    for ct in (0, 1, 2):
        db.compile_file(engine.shipped_fit_path(DT, ct))
    db.compile(tissue.reaction_objects_text(["tt06Endo_fit", "tt06Mid_fit", "tt06Epi_fit"]))
    rm = plugins.ReactionManager(db, list(refgpu.NAMES), DT, t.cell_type, device=local)
    Vm = torch.zeros(t.n, dtype=torch.float64, device="cuda:%d" % local)
    rm.initializeMembraneState(Vm)
    iStim, dVm = torch.zeros_like(Vm), torch.zeros_like(Vm)
    for _ in range(warmup):
        rm.calc(DT, Vm, iStim, dVm)
    torch.cuda.synchronize(local)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(steps):
        rm.calc(DT, Vm, iStim, dVm)
    s1.record()
    s1.synchronize()
    ms = s0.elapsed_time(s1) / steps
    del rm
    ours = {"value": t.n / (ms / 1e3), "ms_per_step": ms}
    ref = {"value": info["cell_steps_per_s"], "ms_per_step": info["ms_per_step"]}
    return {"reference": ref, "ours_plugin": ours, "ours_over_reference": ours["value"] / ref["value"],
            "unit": METRIC, "steps": steps, "warmup": warmup, "dtype": "f64",
            "what": "reaction only (3 BetterTT06 types, Vm and iStim fixed): the reference's NVRTC kernel "
                    "through its ReactionManager::calc, built from its sources with USE_CUDA, against "
                    "plugins.ReactionManager over cdb_reaction_calc (the 6-face GPU diffusion: reference_gpu_diffusion)"}


def reference_gpu_diffusion_block(local, steps=20, warmup=3):
    """The reference's own "cuda" Diffusion on the GPU (CUDADiffusion with
    diff_6face_v1, oracle/_ref/ref_gpu_diff6, in a child process) beside the
    6-face plugin (plugins.CUDADiffusion over cdb_diff6_*): one
    updateLocalVoltage + calc per step, FP64, on a 128 x 120 x 120 box (y
    and z extents multiples of 30, the shapes on which the reference kernel
    reaches every barrier), CUDA events on each side's launching stream; the
    largest difference of the two dVm, relative to the largest |dVm|."""
    from oracle import refgpu
    if not refgpu.diff6_available():
        return None
    import torch
    from cardioid_b200 import plugins, tissue
    t = tissue.box(128, 120, 120, seed=1234)
    ref_dvm, info = refgpu.diff6(t, t.vm0, t.diffusion_scale, steps=steps)
    d = plugins.CUDADiffusion(t, t.diffusion_scale, device=local)
    V = torch.tensor(t.vm0, device="cuda:%d" % local)
    out = torch.empty_like(V)
    for _ in range(warmup):
        d.updateLocalVoltage(V)
        d.calc(out)
    torch.cuda.synchronize(local)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(steps):
        d.updateLocalVoltage(V)
        d.calc(out)
    s1.record()
    s1.synchronize()
    ms = s0.elapsed_time(s1) / steps
    got = out.cpu().numpy()
    d.close()
    ours = {"value": t.n / (ms / 1e3), "ms_per_step": ms}
    ref = {"value": t.n / (info["ms_per_step"] / 1e3), "ms_per_step": info["ms_per_step"]}
    return {"reference": ref, "ours_plugin": ours, "ours_over_reference": ours["value"] / ref["value"],
            "unit": METRIC, "steps": steps, "warmup": warmup, "dtype": "f64", "cells": t.n,
            "max_rel_diff_dvm": float(np.abs(got - ref_dvm).max() / np.abs(ref_dvm).max()),
            "what": "6-face (\"cuda\") diffusion only, 128x120x120 box: the reference's CUDADiffusion (diff_6face_v1, "
                    "map_dVm, copy_to_block) built from its sources, against plugins.CUDADiffusion over cdb_diff6_*"}


def run_reference(args):
    """The reference arm: the reference's own CPU path (oracle/_ref) on the
    same box, timed on the host cores (bench.cpu_baseline); rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args.config)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    cb = cpu_baseline(w, args.steps, args.warmup, args.cpu_omp_steps)
    line = {
        "metric": METRIC, "value": cb["value"], "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic, seeded (no dataset: the configs define geometry, "
                                                     "fibres and pacing)",
        "config": bench_config(w, world),
        "precision": "fp64 (the reference CPU path)",
        "impl": "reference",
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["box256", "box192", "box128", "box64", "shell", "batch4096", "serve"],
                    default="box256")
    ap.add_argument("--shell-dx", type=float, default=0.25)
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--batch-precisions", default="mixed,fp64")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the engine's default tile layout and launch (no timing of the candidates first)")
    ap.add_argument("--jobs", type=int, default=200, help="jobs of --config serve")
    ap.add_argument("--line-jobs", type=int, default=24, help="jobs of the serving block in the headline line")
    ap.add_argument("--rate", type=float, default=5.0, help="job arrivals per second (serving)")
    ap.add_argument("--job-steps", type=int, default=2500,
                    help="steps per served job (0: the full --job-beats paced beats)")
    ap.add_argument("--job-beats", type=int, default=5)
    ap.add_argument("--shell-steps", type=int, default=100, help="timed steps of the shell block in the headline line")
    ap.add_argument("--no-shell", action="store_true", help="skip the shell (config 2) block of the headline line")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving (config 4) block of the headline line")
    ap.add_argument("--serve-batch", type=int, default=250)
    ap.add_argument("--serve-precisions", default="mixed,fp64", help="precisions of --config serve")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--cpu-steps", type=int, default=20, help="steps per CPU slab process (cpu_baseline)")
    ap.add_argument("--cpu-omp-steps", type=int, default=2,
                    help="steps of the one-process omp loop on the whole box (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", choices=["both", "fp64", "mixed"], default="both",
                    help="profiling runs: time one precision only (no headline line)")
    ap.add_argument("--no-e2e", action="store_true", help="profiling runs: skip the end-to-end loop")
    ap.add_argument("--no-apd", action="store_true", help="skip the full-beat APD90 comparison (mixed vs FP64)")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 plugin path")
    ap.add_argument("--stage", type=int, choices=[0, 1, 2, 3], default=None,
                    help="profiling runs: the step kernel's staging mode (default: the engine's)")
    ap.add_argument("--ctas", type=int, default=None, help="profiling runs: CTAs per SM of the persistent grid")
    ap.add_argument("--layout", choices=["cells", "rows"], default=None, help="profiling runs: warp-tile layout")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "shell":
        run_shell(args)
    elif args.config == "batch4096":
        run_batch(args)
    elif args.config == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
