"""Benchmark of the B200 barotropic step.

Workload: the 2048 x 1536 regional basin (1 km, fractal coastline ~40 %
land, log-normal depth, smooth random wind with a 6-hour cycle, dt = 2 s),
FP64.  A step is one leap-frog substep that advances the basin by dt: the
state evolution of barotropic_dynamics(tau=dt, nstep=1) keeping *_e.

  value  grid-cell-steps/s with the state resident in HBM (run_substeps,
         one fused kernel per step), interior cells (land included) x steps,
         summed over ranks; timed with CUDA events on the library's stream.
  e2e    the same metric through the drop-in C-ABI call
         inmsom_barotropic_dynamics(tau = 50*dt, nstep = 50) with pinned host
         buffers: every call uploads the wind forcing RHSx, RHSy (viscosity,
         drag and water flux are registered as static coefficients), runs
         the reference's 2*nstep substeps with time means, and downloads the
         time means.
  cpu_baseline  the CPU oracle (a line-by-line C restatement of the
         reference loops, OpenMP on all host threads) on a bounded sample.

--fp32-velocity measures the same workload with u, up, v, vp stored in FP32
on the device (80 algorithmic bytes per cell and substep; arithmetic, SSH
and budgets FP64); the e2e arm stays FP64.
--study ensemble advances 64 independent regional basins (sides drawn from
192, 256, .., 1536, own seeds, wind amplitude +-20 %) for --steps substeps:
tuned CUDA-graph ensemble, untuned ensemble, and the members one after
another (a study line).
--study closure trains the learned momentum closure on a 2048^2 double-gyre
ridge basin (2 km) coarse-grained to 512^2 (8 km) and compares the
closure-equipped 512^2 run with the plain one (A = 1000 m^2/s) and with
lower plain viscosities: SSH and KE RMSE against the coarse-grained truth
and device time (a study line).
--study closure-kernels times the closure's kernels on the 512^2 coarse basin
with a seeded synthetic state: run_closure against run_substeps (the fused
inference kernel's cost per evaluation) and the training step (gradient +
Adam, batch 65536) (a study line; the ncu summaries use it).
--study baroclinic times the 3-D velocity block of the mode-split step,
inmsom_baroclinic_dynamics (per-column implicit vertical viscosity solve and
Robert-Asselin filter) on the regional basin with --nz s-levels (20) and
seeded synthetic 3-D fields: device time of its kernels with the inputs in
HBM, the end-to-end call with pinned host arrays, the roofline of the
column kernel, a full-size bit-exact check against the CPU oracle and the
oracle's time on the host cores (a study line).
--study tracer times inmsom_tracer_tran_diff (one tracer's transport,
isoneutral/GM diffusion and implicit vertical diffusion) the same way on the
same basin and levels (a study line).
--study general times the per-loop path (the fallback of grids the fused
kernel does not take) on the benchmark basin beside the fused path, and on
the periodic Williamson test-2 sphere (a study line).
--study fp32 runs the FP32-velocity variant against the FP64 run on the
4096 x 4096 ridge basin (2 km, dt = 3 s) for --steps substeps and prints the
per-field max/RMS differences (a study line, not a benchmark line).

--impl reference runs only the CPU oracle arm (rank 0) and prints its line.
Multi-GPU (torchrun): one basin made of N regional basins stacked along y
(2048 x 1536 N), cut into 1 x N row strips, one per rank (weak scaling);
halos of 2*block rows, block substeps per halo exchange (NCCL send/recv of
the packed rows, dist.run_strip); the time is the max over ranks (CUDA
events on each rank's stream) and value sums the ranks' cells.  --replicas
runs independent basins instead; the e2e drop-in call runs one basin per
rank.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "grid-cell-steps/s"
BYTES_PER_CELL_STEP = 120          # algorithmic FP64 bytes of one substep
BYTES_PER_CELL_STEP_F32V = 80      # ... with u, up, v, vp and RHS in FP32
E2E_NSTEP = 50                     # nstep_barotrop of ocean_run.par:9


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10000)
    p.add_argument("--warmup", type=int, default=100)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=2048)
    p.add_argument("--ny", type=int, default=1536)
    p.add_argument("--e2e-calls", type=int, default=12)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--fp32-velocity", action="store_true")
    p.add_argument("--study", default=None,
                   choices=["fp32", "ensemble", "closure", "closure-kernels", "baroclinic", "tracer", "general"])
    p.add_argument("--nz", type=int, default=20, help="s-levels of the baroclinic study")
    p.add_argument("--closure-days", type=float, default=40.0, help="fine spin-up before the training states")
    p.add_argument("--closure-every", type=int, default=10, help="coarse substeps per network evaluation")
    p.add_argument("--closure-tau", type=float, default=0.3, help="wind stress amplitude, N/m^2")
    p.add_argument("--closure-eval", type=int, default=60000, help="coarse substeps of the comparison")
    p.add_argument("--members", type=int, default=64)
    p.add_argument("--group", type=int, default=20)
    p.add_argument("--block", type=int, default=4,
                   help="row strips (--gpus N > 1): substeps per halo exchange (halos of 2*block rows)")
    p.add_argument("--replicas", action="store_true",
                   help="--gpus N > 1: independent basin replicas instead of row strips of one basin")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def workload(args, rank):
    from inmsom_elfs_b200 import basins
    b = basins.regional_basin(nx=args.nx, ny=args.ny, seed=1 + rank)
    return b


def config_dict(b, args, nranks):
    if nranks == 1:
        par = "single"
    elif getattr(args, "replicas", False):
        par = f"replicas{nranks} (independent basins, seed + rank)"
    else:
        par = (f"strips{nranks}: one {b.bounds.nx}x{b.bounds.ny * nranks} basin of {nranks} stacked regional "
               f"basins, 1 x {nranks} row strips, halos of {2 * args.block} rows, {args.block} substeps per "
               f"NCCL halo exchange")
    return {
        "workload": f"regional_basin {b.bounds.nx}x{b.bounds.ny} 1 km FP64 barotropic leap-frog",
        "nx": b.bounds.nx, "ny": b.bounds.ny, "spacing_m": 1000.0, "dt_s": b.dt,
        "land_fraction": round(float(b.info["land_fraction"]), 4),
        "cells_per_rank": b.cells,
        "l2": "inputs larger than L2: 6 state + H + 2 forcing FP64 fields = %.0f MB per step"
              % (9 * 8 * b.cells / 1e6),
        "parallelism": par,
        "step": "one advancing leap-frog substep (barotropic_dynamics(dt,1) state evolution)",
    }


# ------------------------------------------------------------------ clocks
class Clocks:
    """SM clock and clock-event reasons sampled while the timed region runs.

    NVML is polled from a thread every ~1 ms (the timed region of a short
    run lasts a few milliseconds; the library call releases the GIL), the
    device found by its PCI bus id so that CUDA and NVML agree on it; if
    NVML cannot be loaded, nvidia-smi is polled every 100 ms instead.  Only
    reads: no clock or other setting of the GPU is changed."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples = []          # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.proc = None
        self.stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.cuda_index)
        bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus[4:])
        return pynvml, h

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_r = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.bits = [(name, getattr(nv, attr, dflt)) for name, attr, dflt in self.REASONS]

            def poll():
                while not self.stop.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(get_r(h))))
                    except Exception:
                        pass
                    time.sleep(0.001)
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            self.source = "nvml 1 ms"
            return self
        except Exception:
            pass
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.cuda_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
            self.source = "nvidia-smi 100 ms"
        except Exception:
            self.proc = None
        return self

    def _read_smi(self):
        self.bits = [(name, 1 << i) for i, (name, _, _) in enumerate(self.REASONS)]
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz = float(f[1])
                self.max_mhz = float(f[2])
            except ValueError:
                continue
            mask = 0
            for i, v in enumerate(f[5:9]):
                if v.lower().startswith("active"):
                    mask |= 1 << i
            self.samples.append((mhz, mask))

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif getattr(self, "t", None) is not None:
            self.t.join(timeout=2)

    def summary(self):
        sm = [m for m, _ in self.samples]
        reasons = set()
        for _, mask in self.samples:
            for name, bit in getattr(self, "bits", []):
                if mask & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


def gpu_launches(steps: int, fp32_velocity: bool) -> int:
    """Kernels of the timed inmsom_run_substeps(steps) on the fused path:
    one fused kernel per step and one k_advance per replayed graph (graphs
    of min(50, steps rounded down to even) steps); the forcing
    classification (k_minmax3) ran in the warm-up run and is kept, the
    forcing being unchanged.  FP32 velocity storage adds one k_to_f32 (the
    state's velocities; the partner set and the forcing were converted in
    the warm-up run) and one k_vel_from_f32 per run."""
    n = steps
    if steps >= 2:
        n += steps // min(50, steps & ~1)
    if fp32_velocity:
        n += 2
    return n


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the fused kernel from the committed ncu
    summary (scaled to this workload's cells), or None."""
    p = ROOT / "profiles" / "fused_substep_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d


# ------------------------------------------------------------------ CPU arm
def cpu_arm(b, nstep, seconds, threads):
    """Time the oracle's barotropic_dynamics(nstep*dt, nstep) on the host:
    returns (cell-steps/s, calls, elapsed)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as ora
    from inmsom_elfs_b200 import basins
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    ora.barotropic_dynamics(b, nstep * b.dt, nstep)   # warm
    t0 = time.perf_counter()
    calls = 0
    while True:
        ora.barotropic_dynamics(b, nstep * b.dt, nstep)
        calls += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return b.cells * nstep * calls / el, calls, el


def run_reference(args):
    rank, ws, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as ora
    from inmsom_elfs_b200 import basins
    b = workload(args, 0)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    # one call advances nstep steps (2*nstep substeps, the second half for
    # the time means); warm-up and timed calls as many as --warmup and
    # --steps ask for, the timed ones capped at 20 calls (a bounded sample)
    nstep = 5
    for _ in range(max(args.warmup, 0)):
        ora.barotropic_dynamics(b, nstep * b.dt, nstep)
    t0 = time.perf_counter()
    ksteps = max(1, min(args.steps, 20))
    for _ in range(ksteps):
        ora.barotropic_dynamics(b, nstep * b.dt, nstep)
    el = time.perf_counter() - t0
    v = b.cells * nstep * ksteps / el
    cfg = config_dict(b, args, 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        # steps and warmup as run: calls of barotropic_dynamics, each a bounded
        # sample of nstep advancing steps; value and ms_per_step per advancing step
        "steps": ksteps, "warmup": max(args.warmup, 0), "advancing_steps_per_step": nstep,
        "ms_per_step": el / (ksteps * nstep) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{ksteps} calls of the oracle barotropic_dynamics(tau={nstep}*dt, "
                                   f"nstep={nstep}) on the full basin ({2*nstep} substeps per call, "
                                   f"{nstep} advancing steps), OpenMP {threads} threads"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def e2e_arm(args, b, local, barrier, maxall, ws):
    """barotropic_dynamics(E2E_NSTEP*dt, E2E_NSTEP) through the C ABI with
    pinned host arrays, host<->device copies inside the timed region."""
    import torch
    from inmsom_elfs_b200 import solver
    pin = {}
    cells = b.cells
    eb = b.copy()
    for grp in ("state", "means", "forcing", "scratch"):
        d = getattr(eb, grp)
        for k, v in d.items():
            t = torch.empty(v.shape[::-1], dtype=torch.float64, pin_memory=True)
            a = t.numpy().T          # Fortran-contiguous view of pinned memory
            a[...] = v
            d[k] = a
            pin[k] = t
    # INMSOM sets mu and rdis once (Control/init_pars.f90:166-167, 459-481)
    # and the workload's wflux is constant: registered as static coefficients,
    # they are copied in by the first (warm-up) call only
    se = solver.BarotropicSolver(eb, device=local, resident=True, static_coeffs=True)
    se.barotropic_dynamics(E2E_NSTEP * b.dt, E2E_NSTEP)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_calls):
        se.barotropic_dynamics(E2E_NSTEP * b.dt, E2E_NSTEP)
    barrier()
    e2e_s = maxall(time.perf_counter() - t0)
    up, comp, down = se.last_phases()
    se.close()
    fb = 8 * b.bounds.shape[0] * b.bounds.shape[1]
    return {"value": cells * E2E_NSTEP * args.e2e_calls * ws / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": 2 * fb / E2E_NSTEP, "d2h_bytes_per_step": 4 * fb / E2E_NSTEP,
           "ms_per_call": e2e_s / args.e2e_calls * 1e3,
           "last_call_device_ms": {"upload": up, "substeps": comp, "download": down},
           "call": f"inmsom_barotropic_dynamics(tau={E2E_NSTEP}*dt, nstep={E2E_NSTEP}) from pinned "
                   f"host arrays on an INMSOM_RESIDENT | INMSOM_STATIC_COEFFS context: RHSx, RHSy in "
                   f"per call (wflux, mu, rdis stay resident after the warm-up call; mu4 is read only "
                   f"with ksw4 > 0), 4 time-mean arrays out per call, {2 * E2E_NSTEP} substeps with "
                   f"time means; h2d/d2h bytes per advancing step"}



# ------------------------------------------------------------------ GPU arm
def run_ours(args):
    import torch
    rank, ws, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from inmsom_elfs_b200 import basins, solver
    from inmsom_elfs_b200.grid import MEANS

    strips = ws > 1 and not args.replicas
    if strips and args.fp32_velocity:
        raise SystemExit("row strips keep an FP64 state: --fp32-velocity needs --gpus 1 or --replicas")
    if strips:
        # one basin of N stacked regional basins (2048 x 1536 N), one row
        # strip per rank (weak scaling: each rank's strip is basin `rank`),
        # halos of 2k rows, k substeps per NCCL exchange
        from inmsom_elfs_b200.strips import stacked_strip
        parts = {}
        for q in (rank - 1, rank, rank + 1):
            if 0 <= q < ws:
                parts[q] = workload(args, q)
                basins.finalize(parts[q], solver.GpuBackend(local))
        b = stacked_strip(parts, ws, rank, 2 * args.block)
        own = parts[rank]
        del parts
    else:
        b = workload(args, rank)
        basins.finalize(b, solver.GpuBackend(local))
        own = b
    cpu_copy = b.copy() if (rank == 0 and ws == 1 and not args.no_cpu) else None

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def maxall(x):
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident standalone run (value)
    s = solver.BarotropicSolver(b, device=local, resident=True, fp32_velocity=args.fp32_velocity)
    path = s.path()
    s.load_state()
    warm = basins.wind_cycle(args.warmup, b.dt)
    scale = basins.wind_cycle(args.steps, b.dt, t0=args.warmup * b.dt)
    if strips:
        from inmsom_elfs_b200 import dist as sdist
        stepper = sdist.GpuStripStepper(s, host_staging=False)
        sdist.run_strip(stepper, rank, ws, args.warmup, b.dt, warm)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with Clocks(local) as clk:
            ev0.record(stepper.stream)       # the context's stream: the kernels and the exchanges
            sdist.run_strip(stepper, rank, ws, args.steps, b.dt, scale)
            ev1.record(stepper.stream)
            barrier()
        ms = ev0.elapsed_time(ev1)
    else:
        s.run_substeps(args.warmup, b.dt, warm)
        barrier()
        with Clocks(local) as clk:
            ms = s.run_substeps(args.steps, b.dt, scale)
            barrier()
    ms = maxall(ms)
    nbad = s.guard()
    s.close()
    cells = b.cells
    value = cells * args.steps * ws / (ms / 1e3)
    per_launch_s = ms / 1e3 / args.steps
    bpc = BYTES_PER_CELL_STEP_F32V if args.fp32_velocity else BYTES_PER_CELL_STEP
    achieved = bpc * cells / per_launch_s / 1e9
    peak, peak_kind = measured_hbm()

    # ---- e2e through the drop-in with pinned host buffers
    e2e = None
    if not args.no_e2e:
        # the drop-in call is single-domain: with several ranks each runs it
        # on its own regional basin (replicas)
        e2e = e2e_arm(args, own, local, barrier, maxall, ws)

    cpu = None
    if cpu_copy is not None:
        thr = os.cpu_count() or 1
        v, calls, el = cpu_arm(cpu_copy, 5, args.cpu_seconds, thr)
        cpu = {"value": v, "unit": METRIC, "cores": thr, "kind": "port",
               "sample": f"{calls} calls of the oracle barotropic_dynamics(tau=5*dt, nstep=5) on the "
                         f"full basin in {el:.1f} s (10 substeps per call, 5 advancing steps), "
                         f"OpenMP {thr} threads"}

    tr = None if args.fp32_velocity else ncu_traffic()
    traffic = None
    if tr and tr.get("cells"):
        traffic = tr["bytes_per_launch"] * cells / tr["cells"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (u, v stored f32)" if args.fp32_velocity else "f64", "data": "synthetic",
            "config": config_dict(b, args, ws),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_substep (fused leap-frog substep)",
                         "bytes_per_cell_step": bpc,
                         "peak_kind": f"{peak_kind} HBM copy bandwidth"},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "gpu_launches": args.steps + 1 if strips else gpu_launches(args.steps, args.fp32_velocity),
            "path": path[1], "guard_bad_points": nbad,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_study_general(args):
    """The per-loop path (the reference's sweeps, bit-exact rounding) that
    grids the fused kernel does not take -- biharmonic viscosity, periodic
    wraps, ocean halos, metrics varying along rows -- fall back to: device
    time per step on the benchmark basin forced onto it, beside the fused
    path on the same basin, and on the periodic Williamson test-2 sphere
    (which selects it by itself)."""
    import torch
    from inmsom_elfs_b200 import basins, solver
    torch.cuda.set_device(0)
    b = workload(args, 0)
    basins.finalize(b, solver.GpuBackend(0))
    out = {}
    steps = max(args.steps, 2)
    for name, forced in (("fused", False), ("per_loop", True)):
        bg = b.copy()
        with solver.BarotropicSolver(bg, resident=True, force_general=forced) as s:
            s.load_state()
            s.run_substeps(max(args.warmup, 2), b.dt)
            ms = s.run_substeps(steps, b.dt) / steps
            out[name] = {"path": s.path()[1], "ms_per_step": ms, "cell_steps_per_s": b.cells / (ms / 1e3)}
    w = basins.williamson2_basin(1.25, 1.0, backend=solver.GpuBackend(0))
    with solver.BarotropicSolver(w, resident=True) as s:
        s.load_state()
        s.run_substeps(max(args.warmup, 2), w.dt)
        ms = s.run_substeps(steps, w.dt) / steps
        out["williamson2_1.25x1.0"] = {"path": s.path()[1], "cells": w.cells, "ms_per_step": ms,
                                       "cell_steps_per_s": w.cells / (ms / 1e3)}
    out["beta_plane_256"] = beta_plane_256(args)
    print(json.dumps({"study": "general", "workload": f"regional_basin {b.bounds.nx}x{b.bounds.ny} 1 km FP64",
                      "steps": steps, "results": out}), flush=True)


def beta_plane_256(args):
    """The 256 x 256 beta-plane basin (10 km, dt = 15 s: 20 s breaks the
    gravity-wave limit there), 1000 steps: the fused path (L2-resident, so
    bound by launches and the one wave of small work items, not HBM), its
    largest normwise error against the oracle after the 1000 steps, and the
    oracle's own rate on all host threads (barotropic_dynamics calls of 50
    steps)."""
    from oracle import oracle as ora
    from inmsom_elfs_b200 import basins, solver
    nsteps = 1000
    b = basins.beta_plane_basin(n=256)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    bo, bg = b.copy(), b.copy()
    with solver.BarotropicSolver(bg, resident=True) as s:
        s.load_state()
        path = s.path()[1]
        s.run_substeps(max(args.warmup, 2), b.dt)
        s.load_state()
        ms = s.run_substeps(nsteps, b.dt) / nsteps
        s.sync_to_host()
    ora.run_substeps(bo, nsteps, b.dt)
    err = max(float(np.abs(bg.state[k] - bo.state[k]).max() / max(np.abs(bo.state[k]).max(), 1e-300))
              for k in ("ssh_e", "ubrtr_e", "vbrtr_e", "sshp_e", "ubrtrp_e", "vbrtrp_e"))
    threads = os.cpu_count() or 1
    cpu, calls, el = cpu_arm(basins.beta_plane_basin(n=256), 50, min(args.cpu_seconds, 10.0), threads)
    return {"path": path, "cells": b.cells, "steps": nsteps, "dt": b.dt, "ms_per_step": ms,
            "cell_steps_per_s": b.cells / (ms / 1e3), "rel_err_vs_oracle_1000": err,
            "cpu_oracle": {"cell_steps_per_s": cpu, "cores": threads, "sample": f"{calls} calls of 50 steps"}}


def run_study_fp32(args):
    """FP32 velocity storage against the FP64 run on the ridge basin."""
    import torch
    from inmsom_elfs_b200 import basins, solver
    torch.cuda.set_device(0)
    n = 4096 if args.nx == 2048 else args.nx
    b = basins.ridge_basin(n=n)
    basins.finalize(b, solver.GpuBackend(0))
    out, ms, vol = {}, {}, {}
    for fp32 in (False, True):
        bg = b.copy()
        with solver.BarotropicSolver(bg, resident=True, fp32_velocity=fp32) as s:
            s.load_state()
            v0, _ = s.diag()
            ms[fp32] = s.run_substeps(args.steps, b.dt, basins.wind_cycle(args.steps, b.dt))
            v1, e1 = s.diag()
            s.sync_to_host()
        out[fp32], vol[fp32] = bg, (v1 - v0) / v0
    # against the FP64 CPU oracle (the reference's scheme) on a 1024 x 1024
    # part of the same configuration (the oracle would take most of an hour
    # on the 4096 x 4096 basin): both GPU runs' errors per field
    vs_oracle = None
    if not args.no_cpu:
        from oracle import oracle as ora
        nso = 1024 if n > 1024 else n
        so = basins.ridge_basin(n=nso)
        basins.finalize(so, ora.OracleBackend())
        ora.hh_init_external(so)
        steps_o = min(args.steps, 1000)
        sc = basins.wind_cycle(steps_o, so.dt)
        ref = so.copy()
        ora.run_substeps(ref, steps_o, so.dt, sc)
        oc = so.masks["lu"] > 0.5
        vs_oracle = {"workload": f"ridge_basin {nso}x{nso} 2 km dt 3 s", "steps": steps_o, "fields": {}}
        for fp32 in (False, True):
            bg = so.copy()
            with solver.BarotropicSolver(bg, resident=True, fp32_velocity=fp32) as s:
                s.load_state()
                s.run_substeps(steps_o, so.dt, sc)
                s.sync_to_host()
            for k in ref.state:
                d = (bg.state[k] - ref.state[k])[oc]
                r = ref.state[k][oc]
                vs_oracle["fields"].setdefault(k, {})["fp32_velocity" if fp32 else "fp64"] = {
                    "max_abs": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d))),
                    "rel_max": float(np.abs(d).max() / max(np.abs(r).max(), 1e-300))}
    ocean = b.masks["lu"] > 0.5
    errs = {}
    for k in out[False].state:
        a, r = out[True].state[k][ocean], out[False].state[k][ocean]
        d = a - r
        errs[k] = {"max_abs": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d))),
                   "ref_max_abs": float(np.abs(r).max()), "ref_rms": float(np.sqrt(np.mean(r * r))),
                   "rel_max": float(np.abs(d).max() / max(np.abs(r).max(), 1e-300))}
    print(json.dumps({
        "study": "fp32_velocity", "workload": f"ridge_basin {n}x{n} 2 km dt 3 s, wind with a 6 h cycle",
        "steps": args.steps, "fields": errs, "vs_fp64_oracle": vs_oracle,
        "relative_volume_change": {"fp64": vol[False], "fp32_velocity": vol[True]},
        "ms_per_step": {"fp64": ms[False] / args.steps, "fp32_velocity": ms[True] / args.steps},
        "cell_steps_per_s": {"fp64": b.cells * args.steps / (ms[False] / 1e3),
                             "fp32_velocity": b.cells * args.steps / (ms[True] / 1e3)},
    }), flush=True)


def run_study_ensemble(args):
    """64 independent basins: the ensemble as a CUDA graph of one launch per
    member and substep and as one persistent launch per group of substeps
    (tuned and untuned work items), against the members run one after
    another with inmsom_run_substeps."""
    import torch
    from inmsom_elfs_b200 import basins, solver
    torch.cuda.set_device(0)
    rng = np.random.default_rng(1234)
    sides = rng.choice(np.arange(192, 1537, 64), size=args.members)
    amps = rng.uniform(0.8, 1.2, size=args.members)
    bs = []
    for i, (n, a) in enumerate(zip(sides, amps)):
        b = basins.regional_basin(nx=int(n), ny=int(n), seed=100 + i)
        b.taux *= a
        b.tauy *= a
        basins.finalize(b, solver.GpuBackend(0))
        bs.append(b)
    cells = sum(b.cells for b in bs)
    dts = [b.dt for b in bs]
    scale = basins.wind_cycle(args.steps, bs[0].dt)
    solvers = [solver.BarotropicSolver(b, resident=True) for b in bs]
    res = {}
    # members one after another (one launch per substep each)
    for s in solvers:
        s.load_state()
    t = 0.0
    for s, b in zip(solvers, bs):
        s.run_substeps(10, b.dt)
        t += s.run_substeps(args.steps, b.dt, scale)
    res["sequential_members"] = {"ms": t, "cell_steps_per_s": cells * args.steps / (t / 1e3)}
    rows = {}
    with solver.Ensemble(solvers, group=args.group) as e:
        for tag in ("graph_untuned", "persistent_untuned", "graph_tuned", "persistent_tuned"):
            form = tag.split("_")[0]
            e.set_persistent(form == "persistent")
            if tag.endswith("_tuned"):
                rows[form] = e.tune(dts, trial_groups=2)   # each form tuned in that form
            for s in solvers:
                s.load_state()
            e.run(2 * args.group, dts)
            for s in solvers:
                s.load_state()
            ms = e.run(args.steps, dts, scale)
            res[tag] = {"ms": ms, "cell_steps_per_s": cells * args.steps / (ms / 1e3)}
    for s in solvers:
        s.close()
    print(json.dumps({
        "study": "ensemble", "members": args.members, "sides": [int(x) for x in sides],
        "wind_amplitude": [round(float(x), 3) for x in amps], "total_cells": cells, "steps": args.steps,
        "group": args.group, "rows_per_item_chosen": rows, "results": res,
    }), flush=True)


def run_study_closure(args):
    """Learned closure against the plain viscosity on 512^2 coarse-grained
    from 2048^2 (inmsom_elfs_b200.closure.run_study)."""
    import torch
    from inmsom_elfs_b200.closure import ClosureConfig, run_study
    torch.cuda.set_device(0)
    cfg = ClosureConfig(n_coarse=512, factor=4, tau0=args.closure_tau)
    res = run_study(cfg, spinup_days=args.closure_days, snapshots=200, gap=1200, train_steps=20000,
                    eval_gap=20000, eval_steps=args.closure_eval, records=20, every=args.closure_every,
                    extra_plain={"plain_A250": 250.0, "plain_A500": 500.0},
                    log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps({"study": "closure", "data": "synthetic", **res}), flush=True)


def run_study_closure_kernels(args):
    """Timing of the closure kernels (inference fused into the step forcing,
    training step) on the 512^2 coarse basin; synthetic state and data."""
    import torch
    from inmsom_elfs_b200 import _lib, solver
    from inmsom_elfs_b200.closure import ClosureConfig, closure_basins, make_norm
    from inmsom_elfs_b200.mlp import MLP
    torch.cuda.set_device(0)
    cfg = ClosureConfig(n_coarse=512, factor=4)
    b = closure_basins(cfg, solver.GpuBackend(0), which=("base",))["base"]
    bb = b.bounds
    rng = np.random.default_rng(7)
    ocean = b.masks["lu"] > 0.5
    for k, amp in (("ssh_e", 0.02), ("ubrtr_e", 0.1), ("vbrtr_e", 0.1)):
        f = bb.zeros()
        f[bb.interior] = amp * rng.standard_normal((bb.nx, bb.ny))
        b.state[k] = np.asfortranarray(np.where(ocean, f, 0.0))
    b.state["sshp_e"] = b.state["ssh_e"].copy(order="F")
    b.state["ubrtrp_e"] = b.state["ubrtr_e"].copy(order="F")
    b.state["vbrtrp_e"] = b.state["vbrtr_e"].copy(order="F")
    norm = make_norm(b, b.state["ubrtr_e"], b.state["vbrtr_e"], b.state["ssh_e"], out_scale=(1e-9, 1e-9))
    net = MLP(seed=1)
    nsub, res = args.steps - args.steps % 100, {}
    with solver.BarotropicSolver(b) as s:
        s.load_state()
        s.run_substeps(200, cfg.dt_coarse)
        s.run_closure(200, cfg.dt_coarse, 10, net.params.data_ptr(), net.wbf16.data_ptr(), norm)
        t_plain = s.run_substeps(nsub, cfg.dt_coarse)
        res["plain_ms_per_substep"] = t_plain / nsub
        for every in (10, 2):
            s.load_state()
            t = s.run_closure(nsub, cfg.dt_coarse, every, net.params.data_ptr(), net.wbf16.data_ptr(), norm)
            res[f"closure_every{every}_ms_per_substep"] = t / nsub
        per_eval = (res["closure_every2_ms_per_substep"] - res["plain_ms_per_substep"]) * 2
        res["inference_ms_per_evaluation"] = per_eval
        cells = bb.nx * bb.ny
        flop = 2 * (45 * 64 + 64 * 64 + 64 * 2) * cells
        res["inference_cells_per_s"] = cells / (per_eval / 1e3)
        res["inference_tflops"] = flop / (per_eval / 1e3) / 1e12
    n, batch = 1 << 21, 65536
    x = torch.from_numpy(rng.standard_normal((n, 48)).astype(np.float32)).to("cuda").to(torch.bfloat16)
    t = torch.from_numpy(rng.standard_normal((n, 2)).astype(np.float32)).to("cuda")
    net.train(x, t, 20, batch=batch)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    net.train(x, t, 200, batch=batch)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 200
    res["train_ms_per_step"] = ms
    res["train_tflops"] = 3 * 2 * (45 * 64 + 64 * 64 + 64 * 2) * batch / (ms / 1e3) / 1e12
    print(json.dumps({"study": "closure-kernels", "workload": "closure base basin 512x512 8 km, synthetic state",
                      "steps": nsub, "results": res}), flush=True)


BARO_BYTES_PER_CELL_LEVEL = 14 * 8     # 10 nz-level fields read, 4 written (FP64)
BARO_BYTES_PER_COLUMN = 23 * 8 + 2 * 4  # 2-D fields, metrics and the lcu/lcv masks read once


def _pinned_like(a):
    """A pinned host copy of a Fortran-ordered array (same shape and order)."""
    import torch
    t = torch.empty(tuple(reversed(a.shape)), dtype=torch.float64, pin_memory=True)
    out = t.numpy().T
    out[...] = a
    return out


def run_study_baroclinic(args):
    """inmsom_baroclinic_dynamics on the regional basin with nz s-levels."""
    import torch
    from inmsom_elfs_b200 import basins, solver
    torch.cuda.set_device(0)
    b = workload(args, 0)
    basins.finalize(b, solver.GpuBackend(0))
    nz, tau = args.nz, 60.0
    dz, hzt = basins.vertical_grid(nz, 0)
    f = basins.column_fields(b, nz, seed=1, tau=tau)
    names = ("uu", "uup", "vv", "vvp")
    host = {k: _pinned_like(v) for k, v in f.items() if k != "wflux"}
    first = None
    comp, tot = [], []
    clk = Clocks(0)
    with solver.BarotropicSolver(b, resident=False) as s, clk:
        flds = {k: host[k] for k in s.BAROCLINIC_FIELDS}
        st = [host[k] for k in names]
        calls = max(args.steps, 1)
        for it in range(args.warmup + calls):
            for k in names:                       # the same inputs every call
                st[names.index(k)][...] = f[k]
            t0 = time.perf_counter()
            s.baroclinic_dynamics(dz, hzt, tau, *st, **flds)
            wall = (time.perf_counter() - t0) * 1e3
            if first is None:
                first = [a.copy(order="F") for a in st]
            if it >= args.warmup:
                up, cm, dn = s.last_phases()
                comp.append(cm)                   # the kernels' own time (the copies overlap them)
                tot.append(wall)
    cells = b.bounds.nx * b.bounds.ny
    units = cells * nz
    ms = statistics.median(comp)
    ms_e2e = statistics.median(tot)
    alg = units * BARO_BYTES_PER_CELL_LEVEL + cells * BARO_BYTES_PER_COLUMN
    peak, src = measured_hbm()
    tp = ROOT / "profiles" / "k_columns_traffic.json"
    traffic = int(json.loads(tp.read_text())["bytes_per_cell_level"] * units) if tp.exists() else None
    h2d = sum(f[k].nbytes for k in f if k != "wflux") + dz.nbytes + hzt.nbytes
    d2h = sum(f[k].nbytes for k in names)
    line = {
        "study": "baroclinic", "metric": "cell-level-steps/s", "unit": "cell-level-steps/s",
        "value": units / (ms / 1e3), "ms_per_call": ms, "calls": len(comp), "warmup": args.warmup,
        "dtype": "f64", "data": "synthetic (seeded 3-D fields on the regional basin)",
        "config": {"workload": f"baroclinic_dynamics on regional_basin {b.bounds.nx}x{b.bounds.ny}, nz={nz}",
                   "nz": nz, "tau_s": tau, "cells": cells, "land_fraction": round(float(b.info["land_fraction"]), 4),
                   "l2": "inputs larger than L2 (%.1f GB on the device)" % (h2d / 1e9)},
        "e2e": {"value": units / (ms_e2e / 1e3), "unit": "cell-level-steps/s", "ms_per_call": ms_e2e,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "timing": "host wall clock around the C-ABI call (row bands: uploads, solves and downloads "
                          "overlap on three streams)"},
        "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": traffic, "peak_source": src,
                     "traffic_source": "ncu dram bytes of a 512x512x20 launch scaled by cell-levels",
                     "algorithmic_bytes_per_call": int(alg),
                     "kernels_timed": "k_columns (8 row bands) + k_border, CUDA events around each launch"},
        "gpu_launches": 9 * len(comp),            # per call: k_columns for each of 8 row bands, k_border
        "clocks": clk.summary(),
    }
    if not args.no_cpu:
        from oracle import oracle as ora
        threads = os.cpu_count() or 1
        ora.set_threads(threads)
        ref = [f[k].copy(order="F") for k in names]
        t0 = time.perf_counter()
        ora.baroclinic_dynamics(b, dz, hzt, tau, *ref, **{k: f[k] for k in ora.BAROCLINIC_FIELDS})
        el = time.perf_counter() - t0
        line["parity_full_size"] = all(np.array_equal(x, y) for x, y in zip(first, ref))
        line["cpu_baseline"] = {"value": units / el, "unit": "cell-level-steps/s", "cores": threads, "kind": "port",
                                "sample": f"one baroclinic_dynamics call of the same workload ({el:.2f} s)"}
    print(json.dumps(line), flush=True)


TRACER_BYTES_PER_CELL_LEVEL = 14 * 8       # ff ffp uu vv mu src, ww nu and 4 slopes read; ff ffp written
TRACER_BYTES_PER_COLUMN = 15 * 8 + 2 * 4 + 8 * 8   # 2-D inputs and metrics, ig_top/bot, the 8 flux diagnostics


def run_study_tracer(args):
    """inmsom_tracer_tran_diff on the regional basin with nz s-levels."""
    import torch
    from inmsom_elfs_b200 import basins, solver
    torch.cuda.set_device(0)
    b = workload(args, 0)
    basins.finalize(b, solver.GpuBackend(0))
    nz, tau = args.nz, 60.0
    dz, hzt = basins.vertical_grid(nz, 0)
    f = basins.tracer_fields(b, nz, seed=1)
    host = {k: (_pinned_like(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v) for k, v in f.items()}
    shp4 = (*b.bounds.shape, 4)
    fx, fy = _pinned_like(np.zeros(shp4, order="F")), _pinned_like(np.zeros(shp4, order="F"))
    first = None
    comp, tot = [], []
    clk = Clocks(0)
    with solver.BarotropicSolver(b, resident=False) as s, clk:
        for it in range(args.warmup + max(args.steps, 1)):
            host["ff"][...] = f["ff"]
            host["ffp"][...] = f["ffp"]
            t0 = time.perf_counter()
            s.tracer_tran_diff(dz, hzt, tau, host["ff"], host["ffp"], fx, fy, host)
            wall = (time.perf_counter() - t0) * 1e3
            if first is None:
                first = [host["ff"].copy(order="F"), host["ffp"].copy(order="F"), fx.copy(order="F"),
                         fy.copy(order="F")]
            if it >= args.warmup:
                up, cm, dn = s.last_phases()
                comp.append(cm)                   # the kernels' own time (the copies overlap them)
                tot.append(wall)
    cells = b.bounds.nx * b.bounds.ny
    units = cells * nz
    ms, ms_e2e = statistics.median(comp), statistics.median(tot)
    alg = units * TRACER_BYTES_PER_CELL_LEVEL + cells * TRACER_BYTES_PER_COLUMN
    peak, src = measured_hbm()
    h2d = sum(v.nbytes for k, v in f.items() if isinstance(v, np.ndarray)) + dz.nbytes + hzt.nbytes
    d2h = 2 * f["ff"].nbytes + fx.nbytes + fy.nbytes
    line = {
        "study": "tracer", "metric": "cell-level-steps/s", "unit": "cell-level-steps/s",
        "value": units / (ms / 1e3), "ms_per_call": ms, "calls": len(comp), "warmup": args.warmup,
        "dtype": "f64", "data": "synthetic (seeded 3-D fields on the regional basin)",
        "config": {"workload": f"tracer_tran_diff on regional_basin {b.bounds.nx}x{b.bounds.ny}, nz={nz}",
                   "nz": nz, "tau_s": tau, "cells": cells,
                   "l2": "inputs larger than L2 (%.1f GB on the device)" % (h2d / 1e9)},
        "e2e": {"value": units / (ms_e2e / 1e3), "unit": "cell-level-steps/s", "ms_per_call": ms_e2e,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "timing": "host wall clock around the C-ABI call (row bands: uploads, kernels and downloads "
                          "overlap on three streams)"},
        "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": None, "peak_source": src,
                     "algorithmic_bytes_per_call": int(alg),
                     "kernels_timed": "k_tracer_flux, wraps, k_tracer_solve (8 row bands) + k_tracer_border, "
                                      "CUDA events around each band"},
        # per call: k_tracer_flux and k_tracer_solve for each of 8 row bands (and the flux
        # wraps on a periodic basin), k_tracer_border
        "gpu_launches": 17 * len(comp),
        "clocks": clk.summary(),
    }
    if not args.no_cpu:
        from oracle import oracle as ora
        threads = os.cpu_count() or 1
        ora.set_threads(threads)
        ff, ffp = f["ff"].copy(order="F"), f["ffp"].copy(order="F")
        ox, oy = np.zeros(shp4, order="F"), np.zeros(shp4, order="F")
        t0 = time.perf_counter()
        ora.tracer_tran_diff(b, dz, hzt, tau, ff, ffp, ox, oy, f)
        el = time.perf_counter() - t0
        line["parity_full_size"] = all(np.array_equal(x, y) for x, y in zip(first, (ff, ffp, ox, oy)))
        line["cpu_baseline"] = {"value": units / el, "unit": "cell-level-steps/s", "cores": threads, "kind": "port",
                                "sample": f"one tracer_tran_diff call of the same workload ({el:.2f} s)"}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.study == "baroclinic":
        run_study_baroclinic(a)
    elif a.study == "tracer":
        run_study_tracer(a)
    elif a.study == "closure-kernels":
        run_study_closure_kernels(a)
    elif a.study == "closure":
        run_study_closure(a)
    elif a.study == "ensemble":
        run_study_ensemble(a)
    elif a.study == "general":
        run_study_general(a)
    elif a.study == "fp32":
        run_study_fp32(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
