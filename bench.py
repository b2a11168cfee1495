"""Benchmark of the CNRK2 step (ChannelFlow.jl step!, rotational form) on B200.

    python bench.py [--gpus N --steps K --warmup W --config c3 --impl engine|reference]

Workload (default, config "c3"): Re_tau~590-sized Poiseuille at constant bulk
flux, grid 384x257x384, Lx=2pi, Lz=pi, Re_bulk=10900, dt=0.002, seeded
synthetic divergence-free initial state (amplitude 0.1, spectrum
(1+k^2+l^2)^-1 0.8^n), plain FP64.  One "step" is one full three-stage CNRK2
step.  The state (U, P, Q and the nonlinear work fields, >=3.9 GB) is far
larger than the 126 MB L2, so no flush is needed between steps.

The JSON line carries: value (steps/s, device-resident state, CUDA-graph step,
timed with CUDA events on the engine stream, max over ranks), e2e (the same
metric through the host-buffer C-ABI path, cf_step_host: state upload, step,
state download per step from and into pinned memory, the transfers overlapped
with the first and last column kernels), roofline of the dominant kernel (algorithmic
bytes from the fixed byte model / event-timed kernel time), the CPU baseline
(the oracle port on this host's cores, a bounded sample of one CNRK2 stage),
clocks sampled during the timed region, and the kernel-launch count.

N > 1 (torchrun): independent replicas, one per GPU, no data-path collective
(a single channel does not shard; the ensemble of replicas does); the ranks
meet only at the barriers around the timed region and in the maximum of their
times.  --impl reference runs on rank 0 alone.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "channelflow.jl_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = {
    # plain FP64 Couette, Re=400 (c1 of the headline set)
    "c1": dict(Nx=32, Ny=33, Nz=32, Lx=2 * math.pi / 1.14, Lz=2 * math.pi / 2.5, nu=1 / 400, dt=0.01,
               profile="couette", constraint=None, amp=0.1, shape=0, rho=0.8),
    # FP64 Poiseuille at constant flux, Re_bulk=2800
    "c2": dict(Nx=128, Ny=129, Nz=128, Lx=4 * math.pi, Lz=4 * math.pi / 3, nu=(2 / 3) / 2800, dt=0.005,
               profile="poiseuille", constraint=(2 / 3, 0.0), amp=0.2, shape=1, rho=0.7),
    # Re_tau~590-sized Poiseuille at constant flux, Re_bulk=10900 (headline grid)
    "c3": dict(Nx=384, Ny=257, Nz=384, Lx=2 * math.pi, Lz=math.pi, nu=(2 / 3) / 10900, dt=0.002,
               profile="poiseuille", constraint=(2 / 3, 0.0), amp=0.1, shape=1, rho=0.8),
    # ensemble of 256 plane Couette instances on uneven grids (one graph per step)
    "c4": dict(ensemble=[((32, 33, 32), 128), ((48, 49, 48), 96), ((64, 65, 64), 32)],
               Lx=2 * math.pi / 1.14, Lz=2 * math.pi / 2.5, Re=(300.0, 500.0), amp=(0.05, 0.15), dt=0.01,
               profile="couette", constraint=None, shape=0, rho=0.8),
    # large mixed-precision grid 512x385x512 with the state stored in FP32 (FP64
    # Helmholtz, influence-matrix and mean-mode solves); errors against an FP64
    # run of the same 200 steps
    "c5": dict(Nx=512, Ny=385, Nz=512, Lx=2 * math.pi, Lz=math.pi, nu=(2 / 3) / 10900, dt=0.0015,
               profile="poiseuille", constraint=(2 / 3, 0.0), amp=0.1, shape=1, rho=0.8,
               precision="mixed-f32state", err_steps=200),
}
METRIC = "steps/s @384x257x384: mixed vs FP64 plain (<=1e-9 rel err); ensemble agg steps/s"


def sizes(cfg):
    Nxh = cfg["Nx"] // 2 + 1
    Nzp = (3 * cfg["Nz"] + 1) // 2
    Nr = Nxh * cfg["Nz"] * cfg["Ny"]
    Nq = Nxh * Nzp * cfg["Ny"]
    return Nr, Nq


def model_bytes(cfg, s_nl=None, s_state=None):
    """Algorithmic bytes per kernel launch (fixed byte model of the step).

    per stage (rotational form): s_state*14*Nr (U, P, Q read/write) + 16*5*Nr
    (Stokes responses and factors) + s_nl*(18*Nr + 18*Nq) (N read 3, nodes
    written 6, z-inverse 6->6, x-pass 6->3, z-forward 3->3); s_state = s_nl =
    16 for FP64, s_nl = 8 for the mixed forms' FP32 nodal and padded fields,
    s_state = 8 for the FP32 state.  Convective form: z-inverse 6->9, x-pass
    9->3.  Divergence form: nodes written 3, z-inverse 3->3, x-pass 3->6,
    z-forward 6->6, and k_column_div (counted with the column kernel) 6->3.
    """
    prec = cfg.get("precision", "fp64")
    if s_nl is None:
        s_nl = 16 if prec == "fp64" else 8
    if s_state is None:
        s_state = 8 if prec == "mixed-f32state" else 16
    Nr, Nq = sizes(cfg)
    form = cfg.get("form", "rotational")
    if form == "convective":
        return {"zinv": s_nl * (6 * Nr + 9 * Nq), "xpass": s_nl * (12 * Nq), "zfwd": s_nl * (3 * Nq + 3 * Nr),
                "column": 16 * 19 * Nr + s_nl * 9 * Nr}
    if form == "divergence":
        return {"zinv": s_nl * (3 * Nr + 3 * Nq), "xpass": s_nl * (9 * Nq), "zfwd": s_nl * (6 * Nq + 6 * Nr),
                "column": 16 * 19 * Nr + s_nl * 15 * Nr}
    return {
        "zinv": s_nl * (6 * Nr + 6 * Nq),
        "xpass": s_nl * (9 * Nq),
        "zfwd": s_nl * (3 * Nq + 3 * Nr),
        "column": s_state * 14 * Nr + 16 * 5 * Nr + s_nl * 9 * Nr,
    }


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(kernel, cfg_name):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        d = json.load(open(path))
        return d[cfg_name][kernel]
    except Exception:
        return None


def make_oracle(cfg):
    from oracle import oracle as O

    c = cfg
    if c["profile"] == "couette":
        return O.couette(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"], c["nu"], c["dt"])
    return O.poiseuille(c["Nx"], c["Ny"], c["Nz"], c["Lx"], c["Lz"], c["nu"], c["dt"], bulkvelocity=c["constraint"])


def time_oracle_stages(cfg, threads, warmup, count):
    """The oracle port (the reference's algorithm restated in C++) timed on
    this host: full, unsampled CNRK2 stages of the whole workload, `warmup`
    untimed ones, then `count` timed ones (stage j = i mod 3 in turn, as a step
    runs them).  Returns (seconds per step, the stage times): a step is the
    sum over its three stages of the fastest sample of each (the minimum of
    the samples after warm-up, as the reference's own benchmark takes the
    minimum, benchmarks/step.jl:31-53); with fewer than three samples, three
    times the fastest stage."""
    from oracle import oracle as O

    O.set_threads(threads)
    O.set_helmholtz_method("quasitri")
    O.set_sample_div(1)
    c = cfg
    pb = make_oracle(cfg)
    U = pb.synth(seed=1, amp=c["amp"], shape=c["shape"], rho=c["rho"])
    P = pb.zeros()
    pb.prepare()
    for w in range(warmup):
        pb.stage(U, P, w % 3)
    times = [[], [], []]
    for i in range(count):
        j = (warmup + i) % 3
        t0 = time.perf_counter()
        pb.stage(U, P, j)
        times[j].append(time.perf_counter() - t0)
    if all(times):
        step_s = sum(min(t) for t in times)
    else:
        step_s = 3 * min(t for ts in times for t in ts)
    return step_s, times


def cpu_baseline(cfg, name):
    """The CPU baseline of the engine line: one full stage of the workload on
    all host threads after one warm-up stage, and (for the scaling with
    cores) three full stages of 128x129x128 on one thread."""
    threads = os.cpu_count() or 1
    step_s, times = time_oracle_stages(cfg, threads, 1, 1)
    one_s, _ = time_oracle_stages(CONFIGS["c2"], 1, 1, 3)
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"one full CNRK2 stage of {name} ({times[1][0]:.2f} s, after one warm-up stage) on "
                      f"{threads} threads; steps/s = 1/(3 x stage time)",
            "one_thread_c2": {"value": 1.0 / one_s, "unit": "steps/s", "cores": 1,
                              "sample": "three full stages of 128x129x128 (one of each) after one warm-up stage"}}


# ---- replicas: one process per GPU, no data-path collective; the ranks only
# meet at the barriers around the timed region and in the max of their times
def init_ranks(backend="nccl", timeout_s=120):
    """(rank, world, local rank, torch.distributed or None) from the torchrun
    environment; with more than one rank, a process group of `backend` whose
    collectives end with an error after `timeout_s` seconds."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return rank, world, local, None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local, dist


def rank_ops(dist, device="cuda"):
    """barrier() and max_over_ranks(x) of the run (no-ops with one rank); the
    maximum is reduced in a float64 tensor on `device`."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def finish_ranks(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, cfg, rank):
    """--impl reference: the oracle port (the reference's algorithm restated on
    the CPU) on all of this host's cores; each timed step is one full,
    unsampled CNRK2 stage of the workload (time_oracle_stages)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if "ensemble" in cfg:
        members = ensemble_members(cfg, 0)
        cb = ensemble_cpu(cfg, members, threads)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": len(members) / cb["value"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": "c4", "instances": len(members)},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    step_s, times = time_oracle_stages(cfg, threads, args.warmup, args.steps)
    value = 1.0 / step_s
    timed = sum(t for ts in times for t in ts)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.config, **workload_desc(cfg)},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"each timed step is one full, unsampled CNRK2 stage of the workload (stages "
                                   f"0, 1, 2 in turn, {args.warmup} warm-up stages first); steps/s = 1 / (sum over "
                                   f"the three stages of the fastest sample of each); {timed:.1f} s timed"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_desc(cfg):
    return {"grid": [cfg["Nx"], cfg["Ny"], cfg["Nz"]], "Lx": cfg["Lx"], "Lz": cfg["Lz"], "nu": cfg["nu"],
            "dt": cfg["dt"], "profile": cfg["profile"],
            "constraint": ("bulkvelocity" if cfg["constraint"] else "pressuregradient(0,0)"),
            "form": cfg.get("form", "rotational"),
            "precision": ("fp64 plain" if cfg.get("precision", "fp64") == "fp64"
                          else MIXED_DESC[cfg["precision"]]),
            "l2": "state larger than L2 (no flush needed)"}


def ensemble_members(cfg, rank):
    """Members of the ensemble workload: (Nx, Ny, Nz, nu, amplitude, seed),
    Re and amplitude drawn uniformly from the workload's ranges."""
    rng = np.random.default_rng(4 + rank)
    out, i = [], 0
    for (Nx, Ny, Nz), count in cfg["ensemble"]:
        for _ in range(count):
            Re = rng.uniform(*cfg["Re"])
            amp = rng.uniform(*cfg["amp"])
            out.append((Nx, Ny, Nz, 1.0 / Re, amp, 5000 + 1000 * rank + i))
            i += 1
    return out


def ensemble_model_bytes(cfg, members):
    tot = 0.0
    for Nx, Ny, Nz, *_ in members:
        c = dict(cfg, Nx=Nx, Ny=Ny, Nz=Nz)
        tot += 3 * sum(model_bytes(c).values())
    return tot


def run_ensemble(args, cfg, rank, world, local, torch, dist):
    """--config c4: the ensemble line (measure_ensemble) printed by rank 0."""
    line = measure_ensemble(args, cfg, rank, world, local, torch, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_ensemble(args, cfg, rank, world, local, torch, dist):
    """Ensemble workload: value = aggregate steps/s of all instances advanced
    together (cf_step_batch); the same instances stepped one after another,
    each through its own CUDA-graph step, give the sequential figure."""
    import cfb200

    members = ensemble_members(cfg, rank)
    ens = cfb200.Ensemble([dict(grid=cfb200.Grid(Nx, Ny, Nz, cfg["Lx"], cfg["Lz"]), profile="couette", nu=nu,
                                dt=cfg["dt"]) for Nx, Ny, Nz, nu, _, _ in members])
    for inst, (_, _, _, _, amp, seed) in zip(ens.instances, members):
        cfb200.lib().cf_random_state(inst.handle, seed, amp, cfg["shape"], cfg["rho"])
    n = len(members)
    stream = torch.cuda.ExternalStream(ens.stream_ptr())
    barrier, max_over_ranks = rank_ops(dist, "cuda")

    ens.step(args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    launches = ens.launches()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_per_step = ms / args.steps
    value = world * n * args.steps / (ms / 1e3)

    # the same instances one after another, each with its own graph step
    seq_ms = 0.0
    kseq = max(2, min(args.steps, 5))
    for inst in ens.instances:
        s_i = torch.cuda.ExternalStream(inst.stream_ptr())
        inst.advance(0.0, 1)
        inst.sync()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(s_i)
        inst.advance(0.0, kseq)
        a1.record(s_i)
        a1.synchronize()
        seq_ms += a0.elapsed_time(a1) / kseq
    seq_ms = max_over_ranks(seq_ms)
    seq_value = world * n / (seq_ms / 1e3)

    # end to end through the host-buffer C ABI: every instance's state is
    # uploaded from pinned memory and downloaded after each ensemble step
    hb = []
    for inst in ens.instances:
        Uc, Pc = inst.get_state()
        Uh = torch.empty(Uc.shape + (2,), dtype=torch.float64, pin_memory=True).numpy()
        Ph = torch.empty(Pc.shape + (2,), dtype=torch.float64, pin_memory=True).numpy()
        Uh[...] = Uc.view(np.float64).reshape(Uh.shape)
        Ph[...] = Pc.view(np.float64).reshape(Ph.shape)
        hb.append((Uh.view(np.complex128).reshape(Uc.shape), Ph.view(np.complex128).reshape(Pc.shape)))
    ke = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        for inst, (Uv, Pv) in zip(ens.instances, hb):
            inst.set_state(Uv, Pv)
        ens.step(1)
        for inst, (Uv, Pv) in zip(ens.instances, hb):
            U2, P2 = inst.get_state()
            Uv[...] = U2
            Pv[...] = P2
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    state_bytes = sum(4 * 16 * (Nx // 2 + 1) * Nz * Ny for Nx, Ny, Nz, *_ in members)

    peak, peak_kind = peaks()
    mbytes = ensemble_model_bytes(cfg, members)
    achieved = mbytes / (ms_per_step * 1e-3) / 1e9
    energies = [inst.diagnostics()[0] for inst in ens.instances[:: max(1, n // 8)]]
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "c4", "instances": n,
                   "grids": [f"{c}x({g[0]},{g[1]},{g[2]})" for g, c in cfg["ensemble"]],
                   "Re": list(cfg["Re"]), "amp": list(cfg["amp"]), "dt": cfg["dt"], "profile": "couette",
                   "form": "rotational", "precision": "fp64 plain",
                   "l2": "ensemble state (~1.3 GB) larger than L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
        "aggregate": "value = instance-steps/s of the whole ensemble (cf_step_batch, one CUDA graph per step)",
        "sequential": {"value": seq_value, "unit": "steps/s",
                       "how": "the same instances one after another, each through its own CUDA-graph step "
                              "(sum of per-instance event-timed step times)"},
        "speedup_vs_sequential": value / seq_value,
        "e2e": {"value": world * n * ke / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes},
        "roofline": {"bound": "hbm", "kernel": "ensemble step (all kernels, byte model summed over instances)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": None, "step_model_bytes": mbytes},
        "clocks": clocks,
        "gpu_launches": launches,
        "diagnostics": {"kinetic_energy_sample": energies},
        "schedule": [s for s in ens.schedule().splitlines() if s],
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = ensemble_cpu(cfg, members, os.cpu_count() or 1)
    ens.close()
    return line


def ensemble_cpu(cfg, members, threads):
    """Oracle port: one full step of one instance per grid, times the number
    of instances on that grid, summed (instances one after another)."""
    from oracle import oracle as O

    O.set_threads(threads)
    O.set_helmholtz_method("quasitri")
    total = 0.0
    for (Nx, Ny, Nz), count in cfg["ensemble"]:
        nu = next(m[3] for m in members if m[:3] == (Nx, Ny, Nz))
        pb = O.couette(Nx, Ny, Nz, cfg["Lx"], cfg["Lz"], nu, cfg["dt"])
        U, P = pb.random_state(seed=1, amp=0.1)
        pb.step(U, P, 1)
        t0 = time.perf_counter()
        pb.step(U, P, 2)
        total += count * (time.perf_counter() - t0) / 2
    return {"value": len(members) / total, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": "one instance per grid stepped twice on the oracle; ensemble time = sum over grids of "
                      "count x step time; value = instance-steps/s"}


def make_problem(cfb200, g, cfg, precision):
    if cfg["profile"] == "couette":
        return cfb200.CouetteFlow(g, cfg["nu"], cfg["dt"], precision=precision)
    return cfb200.PoiseuilleFlow(g, cfg["nu"], cfg["dt"], bulkvelocity=cfg["constraint"], precision=precision)


MIXED_DESC = {
    "mixed": "FP32 periodic transforms and products (FP32 nodal fields); FP64 Chebyshev transforms, Stokes solve "
             "and state",
    "mixed-tc": "FP32 periodic transforms and products; tensor-core Chebyshev transforms (TF32 heads and "
                "remainders, three products, FP32 accumulation); FP64 Stokes solve and state",
    "mixed-bf16": "FP32 periodic transforms and products; tensor-core Chebyshev transforms (three BF16 pieces per "
                  "operand, six BF16 products, FP32 accumulation); FP64 Stokes solve and state",
    "mixed-f32state": "FP32 periodic transforms and products; velocity, pressure and RK history stored in FP32 "
                      "(widened to FP64 in every stage); FP64 Chebyshev transforms, Helmholtz, influence-matrix, "
                      "mean-mode and flux-constraint solves",
}


def errors_vs_fp64(pb, U0, P0, fp64, nerr):
    """Error of every reported result of problem pb against the FP64 engine
    after nerr steps from (U0, P0) (fp64: fp64_reference_run's result)."""
    Ur, dr, gr = fp64
    pb.set_state(U0, P0)
    _, gm = pb.advance(0.0, nerr)
    Um, _ = pb.get_state()
    dm = pb.diagnostics()

    def rerr(a, b):
        return float(abs(a - b) / max(abs(b), 1e-300))

    return {"steps": nerr,
            "velocity_rel_l2": float(np.linalg.norm(Um - Ur) / np.linalg.norm(Ur)),
            "energy_rel": rerr(dm[0], dr[0]),
            "dissipation_rel": rerr(dm[1], dr[1]),
            "wall_shear_upper_rel": rerr(dm[3], dr[3]),
            "wall_shear_lower_rel": rerr(dm[4], dr[4]),
            "flux_gradient_rel": rerr(gm[0], gr[0]),
            "max_div_mixed": float(dm[2]), "max_div_fp64": float(dr[2])}


def fp64_reference_run(cfg, g, U0, P0, nerr):
    """The FP64 engine's state, diagnostics and last gradients after nerr steps
    from (U0, P0): the reference of the mixed forms' errors."""
    import cfb200

    ref = make_problem(cfb200, g, cfg, "fp64")
    ref.set_state(U0, P0)
    _, grads = ref.advance(0.0, nerr)
    Ur, _ = ref.get_state()
    dr = ref.diagnostics()
    ref.close()
    return Ur, dr, grads


def measure_mixed(args, cfg, g, U0, P0, torch, max_over_ranks, fp64, nerr, precision="mixed"):
    """A mixed-precision step on the same workload: steps/s (device-resident
    state, CUDA-graph step, CUDA events), per-kernel event timing, and the
    error of every reported result against the FP64 step after nerr steps from
    the same initial state (fp64: fp64_reference_run's result).
    precision "mixed": FP32 periodic transforms, FP64 Chebyshev transforms in
    the column kernel; "mixed-tc" / "mixed-bf16": the Chebyshev transforms on
    the tensor cores with the TF32 or the BF16 operand split."""
    import cfb200

    mx = make_problem(cfb200, g, cfg, precision)
    mx.set_state(U0, P0)
    stream = torch.cuda.ExternalStream(mx.stream_ptr())
    mx.advance(0.0, args.warmup)
    mx.sync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    mx.advance(0.0, args.steps)
    launches = mx.launches()
    e1.record(stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    _, kms = mx.advance_profiled(0.0, args.steps)
    nl = 3 * args.steps
    kavg = {"zinv": kms[0] / nl, "xpass": kms[1] / nl, "zfwd": kms[2] / nl, "column": kms[3] / nl,
            "cheb_fwd": kms[4] / nl, "cheb_inv": kms[5] / nl}
    Nr, _ = sizes(cfg)
    Ny, C = cfg["Ny"], 2 * Nr // cfg["Ny"]
    peak, peak_kind = peaks()
    tc_peak = peaks_tensor()
    # tensor-core transform: algorithmic FLOPs of one contraction (2 Ny^2 C per
    # field) and bytes (FP32 in and out); the TF32 split issues 3x the FLOPs
    # (K = 8 per TF32 MMA), the BF16 split 6x (K = 16 at twice the rate)
    cheb = {}
    nprod = {"mixed-tc": 3, "mixed-bf16": 6}.get(precision, 0)
    for key, nf in ((("cheb_fwd", 3), ("cheb_inv", 6)) if nprod else ()):
        t = kavg[key] * 1e-3
        flops, byts = 2.0 * Ny * Ny * C * nf, 8.0 * Ny * C * nf
        cheb[key] = {"ms": kavg[key], "algorithmic_TFLOPs": flops / t / 1e12,
                     "issued_TFLOPs": nprod * flops / t / 1e12, "products": nprod, "GBs": byts / t / 1e9,
                     "hbm_frac": byts / t / 1e9 / peak,
                     # issued rate against the measured dense BF16 peak, halved for
                     # TF32 operands (the TF32 tensor rate is half the BF16 one)
                     "tensor_frac_of_type_peak": ((nprod * flops / t / 1e12) / (tc_peak * (0.5 if nprod == 3 else 1.0))
                                                  if tc_peak else None)}
    out = {"value": args.steps / (ms / 1e3), "unit": "steps/s", "ms_per_step": ms / args.steps,
           "kernel_ms_per_launch": kavg, "gpu_launches": launches,
           "error_vs_fp64": errors_vs_fp64(mx, U0, P0, fp64, nerr),
           "precision": MIXED_DESC[precision]}
    if cheb:
        out["tensor_core_transforms"] = cheb
    mx.close()
    return out


def peaks_tensor():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d.get("bf16_tflops") or 0) or None
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--form", default="rotational", choices=["rotational", "convective", "divergence"],
                    help="nonlinear form of the FP64 step (the mixed form runs the rotational one)")
    ap.add_argument("--err-steps", type=int, default=None,
                    help="steps after which the mixed forms' errors against FP64 are taken (default: the "
                         "configuration's, else 1000)")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed", "mixed-tc", "mixed-bf16", "mixed-f32state"],
                    help="precision of the timed step (default: the configuration's, else fp64)")
    ap.add_argument("--no-c4", action="store_true", help="skip the ensemble measurement of the default line")
    ap.add_argument("--grid", default=None,
                    help="Nx,Ny,Nz replacing the configuration's grid (smaller cases for profiling)")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.grid:
        cfg["Nx"], cfg["Ny"], cfg["Nz"] = (int(v) for v in args.grid.split(","))
    cfg["form"] = args.form
    cfg["precision"] = args.precision or cfg.get("precision", "fp64")
    if args.err_steps is None:
        args.err_steps = cfg.get("err_steps", 1000)
    if args.form != "rotational" or cfg["precision"] != "fp64":
        args.no_mixed = True
    if args.impl == "reference":
        # rank 0 alone times the CPU reference; other ranks exit without work
        run_reference(args, cfg, int(os.environ.get("RANK", "0")))
        return

    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank, world, local, dist = init_ranks("nccl")
    if "ensemble" in cfg:
        run_ensemble(args, cfg, rank, world, local, torch, dist)
        finish_ranks(dist)
        return
    import cfb200

    g = cfb200.Grid(cfg["Nx"], cfg["Ny"], cfg["Nz"], cfg["Lx"], cfg["Lz"])
    prec = cfg["precision"]
    if cfg["profile"] == "couette":
        pb = cfb200.CouetteFlow(g, cfg["nu"], cfg["dt"], form=args.form, precision=prec)
    else:
        pb = cfb200.PoiseuilleFlow(g, cfg["nu"], cfg["dt"], bulkvelocity=cfg["constraint"], form=args.form,
                                   precision=prec)
    cfb200.lib().cf_random_state(pb.handle, 1000 + rank, cfg["amp"], cfg["shape"], cfg["rho"])
    U0, P0 = pb.get_state()
    stream = torch.cuda.ExternalStream(pb.stream_ptr())
    barrier, max_over_ranks = rank_ops(dist, "cuda")

    # warm-up (CUDA-graph step)
    t = 0.0
    t, _ = pb.advance(t, args.warmup)
    pb.sync()

    # ---- timed region: device-resident state, graph-launched steps
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t, _ = pb.advance(t, args.steps)
    launches = pb.launches()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms)
    barrier()
    ms_per_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)

    # ---- per-kernel event timing over the same steps (roofline)
    t, kms = pb.advance_profiled(t, args.steps)
    launches_per_kernel = 3 * args.steps
    kavg = {"zinv": kms[0] / launches_per_kernel, "xpass": kms[1] / launches_per_kernel,
            "zfwd": kms[2] / launches_per_kernel, "column": kms[3] / launches_per_kernel}
    mb = model_bytes(cfg)
    dom = max(kavg, key=kavg.get)
    peak, peak_kind = peaks()
    achieved = mb[dom] / (kavg[dom] * 1e-3) / 1e9
    xname = {"rotational": "k_xpass", "convective": "k_xpass_conv", "divergence": "k_xpass_div"}[args.form]
    knames = {"zinv": "k_zinv", "xpass": xname, "zfwd": "k_zfwd", "column": "k_column_stage"}
    roofline = {"bound": "hbm", "kernel": knames[dom],
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "traffic": (traffic_from_profiles(knames[dom], args.config)
                            if not args.grid and args.form == "rotational" and prec == "fp64" else None),
                "algorithmic_bytes_per_launch": mb[dom],
                "kernel_ms_per_launch": kavg,
                "step_model_bytes": 3 * sum(mb.values()),
                "step_model_frac": 3 * sum(mb.values()) / (ms_per_step * 1e-3) / 1e9 / peak}

    # ---- end to end through the host-buffer C ABI (upload, step, download)
    U_h = torch.empty((3,) + g.spectralsize + (2,), dtype=torch.float64, pin_memory=True).numpy()
    P_h = torch.empty(g.spectralsize + (2,), dtype=torch.float64, pin_memory=True).numpy()
    Uc, Pc = pb.get_state()
    U_h[...] = Uc.view(np.float64).reshape(U_h.shape)
    P_h[...] = Pc.view(np.float64).reshape(P_h.shape)
    Uv = U_h.view(np.complex128).reshape((3,) + g.spectralsize)
    Pv = P_h.view(np.complex128).reshape(g.spectralsize)
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        t = cfb200.step_(pb, Uv, Pv, t, 1)
    f1.record(stream)
    f1.synchronize()
    ems = max_over_ranks(f0.elapsed_time(f1))
    e2e_value = world * args.steps / (ems / 1e3)
    Nr, _ = sizes(cfg)
    state_bytes = 4 * 16 * Nr

    diag = pb.diagnostics()
    # the diagnostics recorded on the device after every step (cf_step_record,
    # no host synchronisation between steps): their cost per evaluation
    krec = max(2, min(args.steps, 5))
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    t, _, _ = pb.advance_recorded(t, krec, 1)
    r1.record(stream)
    r1.synchronize()
    rec_ms = r0.elapsed_time(r1) / krec
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "mixed f32/f64", "data": "synthetic",
        "config": {"workload": args.config, **workload_desc(cfg), "parallelism": f"replicas x{world}"},
        "grid_point_steps_per_s": value * cfg["Nx"] * cfg["Ny"] * cfg["Nz"],
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": launches,
        "diagnostics": {"kinetic_energy": diag[0], "dissipation": diag[1], "max_div": diag[2],
                        "recorded_every_step": {"ms_per_step": rec_ms, "ms_per_evaluation": rec_ms - ms_per_step,
                                                "how": "cf_step_record with every = 1 over %d steps, CUDA events"
                                                       % krec}},
    }
    if prec != "fp64":
        # the timed precision's errors against an FP64 run of the same steps
        fp64 = fp64_reference_run(cfg, g, U0, P0, args.err_steps)
        line["error_vs_fp64"] = errors_vs_fp64(pb, U0, P0, fp64, args.err_steps)
        line["kernel_GBs"] = {k: mb[k] / (kavg[k] * 1e-3) / 1e9 for k in kavg}
    if not args.no_mixed:
        fp64 = fp64_reference_run(cfg, g, U0, P0, args.err_steps)
        line["mixed"] = {}
        for mprec, key in (("mixed", "default"), ("mixed-tc", "tensor_core_tf32"), ("mixed-bf16", "tensor_core_bf16"),
                           ("mixed-f32state", "fp32_state")):
            m = measure_mixed(args, cfg, g, U0, P0, torch, max_over_ranks, fp64, args.err_steps, precision=mprec)
            m["speedup_vs_fp64_plain"] = m["value"] / (value / world)
            line["mixed"][key] = m
    if not args.no_c4 and args.config == "c3" and not args.grid:
        line["c4"] = measure_ensemble(argparse.Namespace(steps=5, warmup=3, no_cpu=True), CONFIGS["c4"], rank,
                                      world, local, torch, dist)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(cfg, args.config)
    if rank == 0:
        print(json.dumps(line), flush=True)
    pb.close()
    finish_ranks(dist)


if __name__ == "__main__":
    main()
