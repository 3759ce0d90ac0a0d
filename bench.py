"""Benchmark of the SNAC explicit step on B200 (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c1|c3|ensemble|adjoint]
    python bench.py --impl reference ...      # the reference's CPU code on the host cores

A "step" is one _AbstractContext_Step of the model (Solve + Sync) over the
whole mesh.  The default workload is the Mohr-Coulomb strain-softening
plastic model of 64 x 32(y) x 64 hex (131,072 hex, 1.31 M tets), synthetic seeded
inputs (snac_b200/workloads.py).  Its state (~0.1 GB) fits in the 126 MB L2,
so a 512 MiB buffer is written between timed steps to flush L2.

Timing: W untimed steps, then K steps, each bracketed by CUDA events
recorded on the library's own stream; barrier + synchronize around the timed
region; the max over ranks is taken.  With --gpus N (torchrun) every rank
advances its own replica of the model (the single-model path is not
sharded): value = all ranks' element-steps / slowest rank's time.

At N = 1 the default line also carries the metric's other forms under
"forms": the small and the largest plain models (c1, 16 x 8(y) x 16 hex;
c3, 128 x 64(y) x 128 hex), the batched
ensemble of 256 models against the same models one launch each, and the
adjoint's cost in forward runs with its finite-difference agreement.

--impl reference times the reference's own hot-path C sources
(oracle/_ref/libsnacref_mt.so: element and node loops on every host CPU,
bitwise equal to the serial build) on the same model in this process.
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
from typing import Optional

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "element-steps/s FP64 plain vs batched vs adjoint cost ratio, 1 B200, at stated tol"
UNIT = "element-steps/s"

# Algorithmic (compulsory) HBM bytes per element-step: persistent state read
# once and written once.  Tet stress 10 x 6 x 8 B x 2 = 960 B; node x and v
# 6 x 8 B x 2 = 96 B per node (nodes per hex below); plastic strain
# 10 x 8 B x 2 = 160 B; per-element parameter 8 B; node temperature 8 B read.
NODES_PER_HEX = {"c1": 2601 / 2048, "c2": 139425 / 131072, "c3": 1081665 / 1048576}


# DRAM bytes (read + write) of one launch of the dominant kernel, from one
# ncu capture of that kernel on the same workload
# (profiles/k_fused_step_plastic_64x32x64.md); None where none was taken.
NCU_TRAFFIC = {("c2", "k_fused_step"): 83.627520e6 + 153.497600e6,
               ("c3", "k_fused_stress"): 657.412352e6 + 1706.645248e6}
# what bounds the dominant kernel instead of HBM, from the same kind of ncu
# capture (fractions of peak; profiles/k_fused_step_plastic_64x32x64.md,
# profiles/k_fused_stress_viscoplastic_128x64x128.md)
NCU_PIPES = {("c2", "k_fused_step"): {"fp64_pipe": 0.384, "issue_active": 0.461, "dram_throughput": 0.175},
             ("c3", "k_fused_stress"): {"fp64_pipe": 0.389, "issue_active": 0.480, "dram_throughput": 0.195}}
# FP64 instructions (thread level: DADD, DMUL, DFMA) of one launch of the
# dominant kernel, from one ncu capture of it on the same workload
# (smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum); None
# where none was taken.  With the device's FP64 rate, measured live by
# snac_gpu_fp64_rate, they give the kernel's FP64 roofline.
NCU_FP64 = {("c2", "k_fused_step"): {"dadd": 382913409, "dmul": 449323008, "dfma": 208497024},
            ("c3", "k_fused_stress"): {"dadd": 3477029944, "dmul": 3983840824, "dfma": 2411197120}}
ARITHMETIC = {
    "c1": "reference rounding (no FMA contraction), bitwise equal to the CPU oracle",
    "c2": "reference rounding (no FMA contraction), bitwise equal to the CPU oracle",
    "c3": "reference operation order without FMA contraction; the Arrhenius viscosity's device log/exp differ "
          "from the reference's libm pow*exp in the last bits (checked against the CPU oracle at 1e-6)",
}


def algorithmic_bytes(workload: str) -> float:
    nph = NODES_PER_HEX[workload]
    b = 960.0 + 96.0 * nph
    if workload in ("c2", "c3"):
        b += 160.0 + 8.0
    if workload == "c3":
        b += 8.0 * nph
    return b


def make_workload(name: str):
    from snac_b200 import workloads as W
    return {"c1": W.c1_elastic, "c2": W.c2_plastic, "c3": W.c3_viscoplastic}[name]()


def fp64_rate():
    """FP64 instructions per second per GPU (independent FMA chains), measured
    on the current device; None if the library cannot run the probe."""
    import ctypes as C
    from snac_b200.context import load_library
    try:
        lib = load_library()
        lib.snac_gpu_fp64_rate.argtypes = [C.POINTER(C.c_double)]
        lib.snac_gpu_fp64_rate.restype = C.c_int
        r = C.c_double(0.0)
        return r.value if lib.snac_gpu_fp64_rate(C.byref(r)) == 0 and r.value > 0 else None
    except (OSError, AttributeError):
        return None


def fp64_roofline(workload: str, kernel: str, kernel_ms: float):
    """The dominant kernel's FP64 instruction rate against the device's."""
    counts = NCU_FP64.get((workload, kernel))
    rate = fp64_rate()
    out = {"peak_inst_per_s": rate, "peak_source": "snac_gpu_fp64_rate (measured in this run)",
           "counts_per_launch": counts, "achieved_inst_per_s": None, "frac": None}
    if counts and rate:
        inst = counts["dadd"] + counts["dmul"] + counts["dfma"]
        out["achieved_inst_per_s"] = inst / (kernel_ms / 1e3)
        out["frac"] = out["achieved_inst_per_s"] / rate
        out["achieved_tflops"] = (counts["dadd"] + counts["dmul"] + 2 * counts["dfma"]) / (kernel_ms / 1e3) / 1e12
        out["peak_tflops"] = 2 * rate / 1e12
    return out


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        try:
            sm = [float(r[1]) for r in self.rows if len(r) >= 9]
            if sm:
                out["sm_mhz"] = statistics.median(sm)
                out["sm_max_mhz"] = max(float(r[2]) for r in self.rows if len(r) >= 9)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            seen = set()
            for r in self.rows:
                for k, nm in enumerate(names):
                    if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                        seen.add(nm)
            out["reasons"] = sorted(seen)
        except Exception:
            pass
        return out


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun env).  The CPU tests run the same
    replica logic with backend="gloo"."""
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, x: float) -> float:
    """Max over ranks (every timing is the slowest rank's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ws: int, units_per_rank: float, seconds_this_rank: float) -> float:
    """Whole-job throughput of ws independent replicas (weak scaling): all
    ranks' units over the slowest rank's time."""
    return ws * units_per_rank / allmax(ws, seconds_this_rank)


# ---------------------------------------------------------------------------------------------
def host_info() -> dict:
    """The host the CPU figures were taken on: logical CPUs and the model name."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


def host_threads() -> int:
    """Host CPUs this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_checker_kind(threads: int) -> str:
    """The reference's own sources when they were compiled here (threaded
    build for more than one thread), else the restatement."""
    from oracle.pyoracle import available
    if threads > 1 and available("reference_mt"):
        return "reference_mt"
    return "reference" if available("reference") else "port"


def cpu_sample(workload: str, threads: int, seconds: float, max_steps: int = 100000):
    """Time the CPU checker on whole SNAC steps of the full workload: the model
    is built and taken through step zero once, then stepped one step at a
    time until `seconds` have passed.  Returns (element-steps/s, kind,
    threads used, steps, seconds)."""
    from oracle.pyoracle import Checker
    kind = cpu_checker_kind(threads)
    cfg = make_workload(workload)
    ck = Checker(cfg, kind, threads=threads)
    ck.time_step_zero()
    ck.step(1)  # first step outside the sample (page-in of the state)
    n, t = 0, 0.0
    while n < max_steps and t < seconds:
        t0 = time.perf_counter()
        rc = ck.step(1)
        t += time.perf_counter() - t0
        n += 1
        if rc != 0:
            raise RuntimeError(f"CPU checker step failed: {ck.last_error()}")
    used = ck.threads
    ck.close()
    return cfg.n_elements * n / t, ("reference" if kind.startswith("reference") else "port"), used, n, t


def run_reference(args, ws, rank):
    """--impl reference: the reference's own hot-path C sources (oracle/_ref,
    the threaded build libsnacref_mt.so: the element and node loops of the
    driver on every host CPU, bitwise equal to the serial build; the
    restatement when the reference could not be compiled) on the same
    workload, in this process.  The model is built and taken through step
    zero once; W warm-up steps, then K steps each timed alone.  Only rank 0
    runs; the other ranks exit without work."""
    if rank != 0:
        return
    try:
        from oracle.pyoracle import Checker
        threads = host_threads()
        kind = cpu_checker_kind(threads)
        w = args.workload if args.workload in ("c1", "c2", "c3") else "c2"
        cfg = make_workload(w)
        ne = cfg.n_elements
        ck = Checker(cfg, kind, threads=threads)
        if ck.time_step_zero() != 0:
            raise RuntimeError(f"step zero failed: {ck.last_error()}")
        if ck.step(args.warmup) != 0:
            raise RuntimeError(f"warm-up failed: {ck.last_error()}")
        per_step = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            rc = ck.step(1)
            per_step.append(time.perf_counter() - t0)
            if rc != 0:
                raise RuntimeError(f"step failed: {ck.last_error()}")
        used = ck.threads
        ck.close()
    except Exception as exc:  # one line either way, never a hang
        print(json.dumps({"impl": "reference", "unavailable": f"CPU reference run failed: {exc}"}), flush=True)
        return
    total = sum(per_step)
    value = ne * args.steps / total
    kind_out = "reference" if kind.startswith("reference") else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, snac_b200/workloads.py)",
        "config": {"workload": workload_name(w), "hex": ne, "tets": ne * 10, "nodes": cfg.n_nodes,
                   "parallelism": f"one model, element and node loops on {used} host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind_out, "host": host_info(),
                         "sample": f"{args.steps} SNAC steps of the full {w} mesh ({ne} hex) after {args.warmup} "
                                   f"warm-up steps, each timed alone; {os.path.basename(PATHS_CPU[kind])}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


PATHS_CPU = {"reference_mt": "oracle/_ref/libsnacref_mt.so", "reference": "oracle/_ref/libsnacref.so",
             "port": "oracle/liboracle.so"}


def workload_name(w):
    return {"c1": "elastic 16x8(y)x16 hex over 100x30x100 km",
            "c2": "Mohr-Coulomb strain-softening 64x32(y)x64 hex over 200x40x200 km, lithostatic IC",
            "c3": "Maxwell visco-plastic + temperature 128x64(y)x128 hex over 400x100x400 km"}[w]


# ---------------------------------------------------------------------------------------------
def run_plain(args, ws, rank, local, workload, with_e2e=True, with_cpu=True):
    """One plain model (c1 / c2 / c3): device-timed steps, the per-kernel
    breakdown and roofline, e2e through the C ABI, the CPU sample.  Returns
    the JSON line (rank 0) or None."""
    import torch
    from snac_b200.context import SnacContext

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfg = make_workload(workload)
    ne = cfg.n_elements
    ctx = SnacContext(cfg)
    ctx.time_step_zero()
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # warm-up (also captures the CUDA graphs)
    ctx.step(max(2, args.warmup))
    torch.cuda.synchronize()

    # ---- device-timed steps ------------------------------------------------------------
    # each step: a 512 MiB write that evicts the model state from L2, then the
    # step's graph between two CUDA events on the library's stream; the
    # status is read once after the K steps (snac_gpu_time_steps)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.5)
    l0 = ctx.launches
    barrier(ws)
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    step_ms = ctx.time_steps(args.steps, flush.data_ptr(), flush.numel() * flush.element_size())
    torch.cuda.synchronize()
    barrier(ws)
    wall = time.perf_counter() - wall0
    launches = ctx.launches - l0
    clocks = sampler.stop() if sampler else None
    t_dev = sum(step_ms) / 1e3
    value = replica_throughput(ws, ne * args.steps, t_dev)

    # ---- per-kernel breakdown: one step kernel by kernel, events on the library stream -----
    kern = {}
    nb = max(3, min(10, args.steps))
    for _ in range(nb):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        for name, ms in ctx.profile_step():
            kern.setdefault(name, []).append(ms)
    kern_ms = {k: statistics.mean(v) for k, v in kern.items()}
    top = max(kern_ms, key=kern_ms.get)
    peak, peak_kind = load_peaks()
    alg = algorithmic_bytes(workload)
    step_ms_mean = 1e3 * t_dev / args.steps
    achieved_step = alg * ne / (step_ms_mean / 1e3) / 1e9
    kb = KERNEL_BYTES.get(top, lambda w: alg)(workload)
    achieved_kernel = kb * ne / (kern_ms[top] / 1e3) / 1e9

    # ---- end to end through the C ABI with host buffers --------------------------------
    e2e = None
    if with_e2e and not args.no_e2e:
        from snac_b200.abi import State
        st = ctx.state()
        # the model's state, what one step reads and writes: coordinates, velocities,
        # stresses, and the plugins' per-tet / per-node state (plastic strain,
        # temperature, the Drucker-Prager tensor) where the model has them
        fields = ["coord", "velocity", "stress"]
        if cfg.plugin in ("SnacPlastic", "SnacViscoPlastic"):
            fields.append("plastic_strain")
        if cfg.temperature:
            fields.append("temperature")
        if ctx.keeps_plastic_strain_tensor:
            fields.append("plastic_strain_tensor")
        host = State.empty(ctx.ne, ctx.nn)
        out = State.empty(ctx.ne, ctx.nn)       # the step's result, into pinned host buffers
        keep = []
        for f, _ in out.view()._fields_:
            if f in fields:
                t = torch.from_numpy(getattr(st, f)).pin_memory()
                keep.append(t)
                setattr(host, f, t.numpy())
                t = torch.from_numpy(getattr(out, f)).pin_memory()
                keep.append(t)
                setattr(out, f, t.numpy())
            else:
                setattr(host, f, None)
                setattr(out, f, None)
        h2d = sum(getattr(host, f).nbytes for f in fields)
        d2h = sum(getattr(out, f).nbytes for f in fields)
        ke = max(3, min(args.steps, 10))
        ctx.step_host(host, out, fields, fields)  # first call: the slab streams and staging
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            # host -> device (the step's inputs), one step, device -> host (its result),
            # overlapped slab by slab
            ctx.step_host(host, out, fields, fields)
        torch.cuda.synchronize()
        te = (time.perf_counter() - t0) / ke
        # the same transfers as three calls in sequence, for comparison
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            ctx.set_state(host, fields)
            ctx.step(1)
            ctx.state(out)
        torch.cuda.synchronize()
        t3 = (time.perf_counter() - t0) / ke
        e2e = {"value": ws * ne / allmax(ws, te), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "three_calls": ws * ne / allmax(ws, t3),
               "note": "per step: snac_gpu_step_host with the state (" + ", ".join(fields) + ") in pinned host "
                       "buffers: upload, one step and download overlapped slab by slab; three_calls: "
                       "snac_gpu_upload, snac_gpu_step(1), snac_gpu_download in sequence"}

    ctx.close()
    cpu = None
    if with_cpu and rank == 0 and ws == 1 and not args.no_cpu:  # the CPU sample is taken at N = 1 only
        cpu = cpu_baseline(workload, ne, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_mean, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, snac_b200/workloads.py)",
            "config": {"workload": workload_name(workload), "hex": ne, "tets": ne * 10, "nodes": cfg.n_nodes,
                       "l2": "512 MiB flush written between timed steps",
                       "parallelism": "replicas" if ws > 1 else "single model",
                       "arithmetic": ARITHMETIC[workload]},
            "roofline": {"bound": "hbm", "achieved": achieved_kernel, "peak": peak, "unit": "GB/s",
                         "frac": achieved_kernel / peak, "traffic": NCU_TRAFFIC.get((workload, top)),
                         "kernel": top, "ncu_pipes": NCU_PIPES.get((workload, top)),
                         "fp64": fp64_roofline(workload, top, kern_ms[top]),
                         "kernel_ms": kern_ms[top], "algorithmic_bytes_per_hex": kb,
                         "peak_source": peak_kind,
                         "step": {"achieved": achieved_step, "frac": achieved_step / peak,
                                  "algorithmic_bytes_per_hex": alg}},
            "kernels_ms": kern_ms,
            "gpu_launches": int(launches),
            "wall_s": wall,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        return line
    return None


def verbatim_bc_cost(seconds: float) -> Optional[dict]:
    """The cost of the reference's boundary-condition lookup on the elastic
    16x8x16 workload, one core: StGermain's VariableCondition_ApplyToIndex
    searches the condition's index table linearly for every node and step
    (VariableCondition.c:449-463); the checkers (and the baselines above) use
    an O(1) per-node mask with the same results.  None without the compiled
    reference."""
    from oracle.pyoracle import Checker
    if cpu_checker_kind(1) != "reference":
        return None
    cfg = make_workload("c1")
    out = {}
    for name, on in (("mask", False), ("verbatim", True)):
        ck = Checker(cfg, "reference")
        ck.set_verbatim_bc(on)
        ck.time_step_zero()
        ck.step(1)
        n, t = 0, 0.0
        while t < seconds / 2:
            t0 = time.perf_counter()
            if ck.step(1) != 0:
                raise RuntimeError(ck.last_error())
            t += time.perf_counter() - t0
            n += 1
        ck.close()
        out[name] = cfg.n_elements * n / t
    return {"workload": "elastic 16x8(y)x16 hex", "unit": UNIT, "mask": out["mask"], "verbatim": out["verbatim"],
            "slowdown": out["mask"] / out["verbatim"]}


def cpu_baseline(workload: str, ne: int, args) -> dict:
    """The reference's own sources on the host: all host threads (the
    headline CPU figure) and one core, each a time-boxed sample of whole
    steps of the full mesh."""
    v, kind, used, n, t = cpu_sample(workload, host_threads(), args.cpu_seconds)
    v1, _, _, n1, t1 = cpu_sample(workload, 1, args.cpu_seconds_one)
    return {"value": v, "unit": UNIT, "cores": used, "kind": kind, "host": host_info(),
            "sample": f"{n} SNAC steps of the full {workload} mesh ({ne} hex) on {used} host threads "
                      f"(element and node loops split across them), {t:.1f} s",
            "one_core": {"value": v1, "unit": UNIT, "steps": n1, "seconds": round(t1, 2)},
            "verbatim_bc": verbatim_bc_cost(4.0)}


# Algorithmic bytes per hex of one launch of each kernel (state it must read / write once).
KERNEL_BYTES = {
    "k_fused_step": lambda w: 960.0 + 48.0 * NODES_PER_HEX[w] + (160.0 + 8.0 if w != "c1" else 0.0),
    "k_calc_stresses": lambda w: 960.0 + 48.0 * NODES_PER_HEX[w] + (160.0 + 8.0 if w != "c1" else 0.0)
                                 + (8.0 * NODES_PER_HEX[w] if w == "c3" else 0.0),
    "k_fused_stress": lambda w: 960.0 + 48.0 * NODES_PER_HEX[w] + (160.0 + 8.0 if w != "c1" else 0.0)
                                + (8.0 * NODES_PER_HEX[w] if w == "c3" else 0.0),
    "k_loop_nodes": lambda w: 480.0 + 96.0 * NODES_PER_HEX[w],
    "k_update_elements": lambda w: 960.0 + 48.0 * NODES_PER_HEX[w],
}


# ---------------------------------------------------------------------------------------------
def run_ensemble(args, ws, rank, local, with_e2e=True, with_cpu=True):
    """--workload ensemble: 256 independent plastic / visco-plastic models of
    uneven size advanced together (one launch per kernel type per step),
    against the same models stepped one launch each (each model's own
    step graph, back to back on the same stream)."""
    import torch
    from snac_b200 import workloads as W
    from snac_b200.abi import State
    from snac_b200.batch import SnacBatch, autotune

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfgs = W.c4_ensemble()
    b = SnacBatch(cfgs)
    ne = b.n_elements
    b.time_step_zero()
    tuning = autotune(b, steps=8)
    b.step(max(3, args.warmup, tuning["steps_per_graph"]))  # warm-up; captures the graphs
    torch.cuda.synchronize()

    # state of all models: ~7 GB, far above the 126 MB L2, so no flush is needed
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.5)
    l0 = b.launches
    barrier(ws)
    torch.cuda.synchronize()
    ms = b.time_steps(args.steps)
    launches = b.launches - l0
    b.time_steps(4, each=True)  # captures the per-model graphs (both parities, heat flux formed or not)
    ms_each = b.time_steps(max(3, args.steps // 4), each=True) * args.steps / max(3, args.steps // 4)
    barrier(ws)
    clocks = sampler.stop() if sampler else None
    value = replica_throughput(ws, ne * args.steps, ms / 1e3)
    value_each = ws * ne * args.steps / allmax(ws, ms_each / 1e3)

    peak, peak_kind = load_peaks()
    alg_total = 0.0
    for c in cfgs:
        nph = c.n_nodes / c.n_elements
        alg_total += c.n_elements * (960.0 + 96.0 * nph + 160.0 + 8.0 + (8.0 * nph if c.temperature else 0.0))
    achieved = alg_total / (ms / 1e3 / args.steps) / 1e9

    # end to end: every model's state up from pinned host memory, one batched
    # step, every model's state down, per step
    e2e = None
    if with_e2e and not args.no_e2e:
        def state_fields(m):  # a model's state: what one step reads and writes
            f = ["coord", "velocity", "stress"]
            if m.cfg.plugin in ("SnacPlastic", "SnacViscoPlastic"):
                f.append("plastic_strain")
            if m.cfg.temperature:
                f.append("temperature")
            return f

        hosts, outs = [], []
        for m in b.models:
            st = m.state()
            fl = state_fields(m)
            h, o = State.empty(m.ne, m.nn), State.empty(m.ne, m.nn)
            for f, _ in h.view()._fields_:
                setattr(h, f, torch.from_numpy(getattr(st, f)).pin_memory().numpy() if f in fl else None)
                setattr(o, f, torch.from_numpy(getattr(o, f)).pin_memory().numpy() if f in fl else None)
            hosts.append((h, fl))
            outs.append(o)
        h2d = sum(getattr(h, f).nbytes for h, fl in hosts for f in fl)
        d2h = h2d
        ke = 2
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            for m, (h, fl) in zip(b.models, hosts):
                m.set_state(h, fl)
            b.step(1)
            for m, o in zip(b.models, outs):
                m.state(o)
        torch.cuda.synchronize()
        te = (time.perf_counter() - t0) / ke
        e2e = {"value": ws * ne / allmax(ws, te), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "note": "per step: snac_gpu_upload of every model's state from pinned host buffers, "
                       "snac_gpu_batch_step(1), snac_gpu_download of every model's state"}

    cpu = None
    if with_cpu and rank == 0 and ws == 1 and not args.no_cpu:  # the CPU sample is taken at N = 1 only
        # the first 8 models one after another, each on all host threads
        from oracle.pyoracle import Checker
        threads = host_threads()
        kind = cpu_checker_kind(threads)
        t = 0.0
        hexsteps = 0
        used = 1
        for c in cfgs[:8]:
            ck = Checker(c, kind, threads=threads)
            ck.time_step_zero()
            ck.step(1)
            t0 = time.perf_counter()
            ck.step(16)
            t += time.perf_counter() - t0
            hexsteps += 16 * c.n_elements
            used = ck.threads
            ck.close()
        cpu = {"value": hexsteps / t, "unit": UNIT, "cores": used,
               "kind": "reference" if kind.startswith("reference") else "port", "host": host_info(),
               "sample": f"16 SNAC steps of each of the first 8 ensemble models ({hexsteps // 16} hex), one model "
                         f"after another on {used} host threads, {t:.1f} s"}
    b.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, snac_b200/workloads.py)",
            "config": {"workload": "batched ensemble: 256 models, hex per model drawn in [8..48] x [4..24](y) x "
                                   "[8..48], half Mohr-Coulomb plastic, half visco-plastic with a geotherm",
                       "hex": ne, "models": len(cfgs), "tuning": tuning,
                       "l2": "inputs larger than L2 (~7 GB of model state)",
                       "parallelism": "replicas" if ws > 1 else "single GPU, one launch per kernel type per step"},
            "one_launch_each": {"value": value_each, "ms_per_step": ms_each / args.steps,
                                "speedup_of_batched": value / value_each},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "whole batched step",
                         "algorithmic_bytes_per_step": alg_total, "peak_source": peak_kind},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        return line
    return None


# ---------------------------------------------------------------------------------------------
def run_adjoint(args, ws, rank, local):
    """--workload adjoint: the visco-plastic adjoint workload (32 x 16(y) x 32
    hex, constant dt, fixed uniform temperature), loss = top-surface v_y and
    topography misfit after `--adj-steps` steps against a run with smooth
    +-10 % cohesion and viscosity perturbations; gradients with respect to
    the per-element cohesion, friction and viscosity scales, checkpoint
    every 45 steps.

    Reports (1) the adjoint's cost in forward runs on that workload as
    configured (FLAC damping 0.8), and (2) agreement with central finite
    differences of GPU forward runs: over the full horizon with the
    damping off, and over 24 steps with it on.  With the damping on, the
    loss is discontinuous in the parameters wherever a nodal velocity
    changes sign (the damping force jumps by 2 demf |F|) and the tangent
    dynamics grow exponentially, so no exact gradient can match finite
    differences over thousands of steps."""
    import numpy as np
    import torch
    from snac_b200 import workloads as W
    from snac_b200.adjoint import adjoint, forward_loss, top_surface
    from snac_b200.context import SnacContext

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nx, ny, nz, N, K = 32, 16, 32, args.adj_steps, 45
    ne = nx * ny * nz
    ones = np.ones(ne)

    def maker(demf):
        def make(c, f, v):
            cfg = W.c5_adjoint(nx, ny, nz, t_uniform=300.0)
            cfg.demf = demf
            cfg.element_cohesion_scale, cfg.element_friction_scale, cfg.element_visc_scale = c, f, v
            return cfg
        return make

    def problem(make, n):
        with SnacContext(make(1.0 + W.smooth_field(nx, ny, nz, 7), ones, 1.0 + W.smooth_field(nx, ny, nz, 8))) as t:
            t.time_step_zero()
            t.step(n)
            tv, ty = top_surface(t.cfg, t.state())
        return tv, ty, 1.0 / max(1e-30, float(np.mean(tv ** 2))), 1.0 / (20.0e3 ** 2)

    p = (ones.copy(), ones.copy(), 1.0 + 0.05 * np.random.default_rng(2).uniform(-1, 1, ne))

    def fd_check(make, n, h, ndir, seed):
        tv, ty, wv, wh = problem(make, n)
        with SnacContext(make(*p)) as ctx:
            ctx.time_step_zero()
            r = adjoint(ctx, n, tv, ty, wv, wh, checkpoint_every=K)
        g = [r.grad["cohesion"], r.grad["friction"], r.grad["viscosity"]]
        rng = np.random.default_rng(seed)
        errs = []
        for _ in range(ndir):
            d = [rng.standard_normal(ne) for _ in range(3)]
            lp = forward_loss(make, *[x + h * dx for x, dx in zip(p, d)], n, tv, ty, wv, wh)
            lm = forward_loss(make, *[x - h * dx for x, dx in zip(p, d)], n, tv, ty, wv, wh)
            fd = (lp - lm) / (2 * h)
            ad = sum(float(np.dot(x, y)) for x, y in zip(g, d))
            errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
        return errs

    make = maker(0.8)
    tv, ty, wv, wh = problem(make, N)
    # forward alone: N steps from step zero, device time
    with SnacContext(make(*p)) as ctx:
        ctx.time_step_zero()
        stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
        ctx.step(N)
        with torch.cuda.stream(stream):
            b.record(stream)
        torch.cuda.synchronize()
        ms_fwd = a.elapsed_time(b)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.5)
    with SnacContext(make(*p)) as ctx:
        ctx.time_step_zero()
        l0 = ctx.launches
        t0 = time.perf_counter()
        r = adjoint(ctx, N, tv, ty, wv, wh, checkpoint_every=K)
        wall = time.perf_counter() - t0
        launches = ctx.launches - l0
    clocks = sampler.stop() if sampler else None
    ms_adj = r.ms_forward + r.ms_reverse
    gnorm = float(max(np.abs(r.grad[k]).max() for k in r.grad))
    fd_long = fd_check(maker(0.0), N, 1.0e-5, args.adj_fd, 11) if args.adj_fd else []
    fd_short = fd_check(make, 24, 1.0e-6, args.adj_fd, 12) if args.adj_fd else []
    if rank == 0:
        value = ne * N / (ms_adj / 1e3)
        line = {
            "metric": METRIC, "value": value, "unit": "element-steps/s (forward + adjoint)", "n_gpus": ws,
            "steps": N, "warmup": 0, "ms_per_step": ms_adj / N, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, snac_b200/workloads.py)",
            "config": {"workload": "adjoint: visco-plastic 32x16(y)x32 hex, constant dt, fixed uniform temperature, "
                                   "top-surface v_y + topography misfit, gradients w.r.t. per-element cohesion, "
                                   "friction, viscosity scales", "hex": ne, "checkpoint_every": r.checkpoint_every,
                       "checkpoints": r.checkpoints, "demf": 0.8},
            "adjoint": {"loss": r.loss, "ms_forward_alone": ms_fwd, "ms_adjoint_call": ms_adj,
                        "ms_adjoint_forward_sweep": r.ms_forward, "ms_adjoint_reverse": r.ms_reverse,
                        "cost_in_forward_runs": ms_adj / ms_fwd, "max_abs_gradient": gnorm,
                        "fd_full_horizon_demf0": {"steps": N, "h": 1.0e-5, "rel_errs": fd_long,
                                                  "max": max(fd_long) if fd_long else None},
                        "fd_24_steps_demf08": {"steps": 24, "h": 1.0e-6, "rel_errs": fd_short,
                                               "max": max(fd_short) if fd_short else None}},
            "gpu_launches": int(launches), "wall_s": wall, "clocks": clocks, "e2e": None, "cpu_baseline": None,
        }
        return line
    return None


def run_forms(args, ws, rank, local) -> dict:
    """The metric's other forms beside the headline plain model, each on the
    same GPU in the same run: the small and the largest plain models (c1,
    c3), the batched ensemble against the same models one launch each, and
    the adjoint's cost in forward runs with its finite-difference agreement.
    A form that fails reports its error instead of ending the run."""
    import torch
    forms = {}

    def guarded(name, fn):
        try:
            forms[name] = fn()
        except Exception as exc:  # the headline line is printed either way
            forms[name] = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    def plain(workload):
        ln = run_plain(args, ws, rank, local, workload, with_e2e=True, with_cpu=False)
        return {k: ln[k] for k in ("value", "unit", "ms_per_step", "config", "roofline", "kernels_ms", "gpu_launches",
                                   "clocks", "e2e")}

    def batched():
        ln = run_ensemble(args, ws, rank, local, with_e2e=False, with_cpu=False)
        out = {k: ln[k] for k in ("value", "unit", "ms_per_step", "config", "one_launch_each", "roofline",
                                  "gpu_launches", "clocks")}
        out["speedup_of_batched"] = ln["one_launch_each"]["speedup_of_batched"]
        return out

    def adjoint_form():
        ln = run_adjoint(args, ws, rank, local)
        out = {k: ln[k] for k in ("value", "unit", "steps", "ms_per_step", "config", "adjoint", "gpu_launches",
                                  "clocks")}
        out["cost_in_forward_runs"] = ln["adjoint"]["cost_in_forward_runs"]
        return out

    guarded("plain_c1", lambda: plain("c1"))
    guarded("plain_c3", lambda: plain("c3"))
    guarded("batched", batched)
    guarded("adjoint", adjoint_form)
    return forms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "ensemble", "adjoint"])
    ap.add_argument("--no-forms", action="store_true",
                    help="c2 at N = 1 only: skip the c3, batched and adjoint forms added to the line")
    ap.add_argument("--adj-steps", type=int, default=2000)
    ap.add_argument("--adj-fd", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="time box of the all-threads CPU sample (whole steps)")
    ap.add_argument("--cpu-seconds-one", type=float, default=5.0,
                    help="time box of the one-core CPU sample (whole steps)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, ws, rank)
        return
    ws, rank, local = dist_setup()
    try:
        if args.workload == "ensemble":
            line = run_ensemble(args, ws, rank, local)
        elif args.workload == "adjoint":
            line = run_adjoint(args, ws, rank, local)
        else:
            line = run_plain(args, ws, rank, local, args.workload)
            # the batched and adjoint forms of the metric ride on the default
            # line; under torchrun every rank skips them alike
            if args.workload == "c2" and ws == 1 and not args.no_forms:
                line["forms"] = run_forms(args, ws, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
