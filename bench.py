#!/usr/bin/env python
"""Throughput of the B200 direct Fock build + two-electron nuclear gradient.

One step = one direct J/K build plus one two-electron gradient evaluation on
the same density, for the 40-atom RHF/6-31G* workload (392 Cartesian basis
functions, d shells up to (dd|dd) at Rys order 5; seeded synthetic molecule,
converged RHF density from an SCF run with this library before timing).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl iqcp|reference]

Under torchrun every rank runs an independent replica on its own GPU (the
path has no exchange step); rank 0 prints one JSON line.  ``--impl reference``
times the reference algorithm's CPU restatement (the oracle; the reference's
Rust code cannot be built here) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Fock J/K builds/s + gradient evals/s, mixed vs FP64 at ≤1 µHa / ≤1e-6 Ha/bohr"
UNIT = "steps/s (1 J/K build + 1 gradient eval)"
WORKLOAD = "c2"
L2_FLUSH_BYTES = 256 << 20
MIXED_CUTOFF = 1e-3          # Schwarz x density bound below which quartets run in FP32
BATCH_SIZE = 64              # geometries of the batched measurement (8-48 atoms, H-Cl, 6-31G*)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="iqcp", choices=["iqcp", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample-stride", type=int, default=16,
                    help="oracle CPU baseline evaluates every stride-th bra shell pair")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=BATCH_SIZE,
                    help="geometries in the batched measurement (0: skip)")
    ap.add_argument("--modes", default="",
                    help="force kernel variants instead of autotuning, e.g. 'jk:0,grad:1' (for profiling runs)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-form measurement")
    ap.add_argument("--batch-scf", action="store_true",
                    help="also run the batched device SCF + gradients to convergence")
    return ap.parse_args()


def max_over_ranks(x, world):
    """Largest value of x over the ranks (every rank calls this, in the same
    order); the job's time is the slowest replica's."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, seconds):
    """Whole-job steps/s: each of `world` replicas runs `steps` steps in at most `seconds`."""
    return world * steps / seconds


def workload_config(b, seed):
    return {"workload": "40-atom C/N/O/H molecule, RHF/6-31G* (%d Cartesian bf, %d shells), seed %d"
                        % (b.n_basis, b.n_shells, seed),
            "basis": "6-31g*", "n_atoms": int(b.n_atoms), "nbf": int(b.n_basis),
            "step": "1 direct J/K build + 1 two-electron gradient, converged RHF density",
            "screening": "Schwarz 1e-12, primitive K 1e-15",
            "l2": "flushed between timed steps (256 MiB device write)"}


def cpu_baseline(b, D, stride, phase=0):
    """Oracle (the reference algorithm restated in C++) on every stride-th bra
    shell pair, all host threads; scaled to the full workload."""
    import oracle
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    _, _, cnt = oracle.jk_direct(b, D, stride, phase)
    t1 = time.perf_counter()
    oracle.eri_gradient(b, D, 1.0, stride, phase)
    t2 = time.perf_counter()
    t_step = (t1 - t0) * stride + (t2 - t1) * stride
    return {"value": 1.0 / t_step, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "every %d-th bra shell pair of the same workload (J/K %.1f s + gradient %.1f s of CPU "
                      "wall time, scaled by %d)" % (stride, t1 - t0, t2 - t1, stride),
            "jk_s": (t1 - t0) * stride, "grad_s": (t2 - t1) * stride}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.3 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


def timed_steps(step, steps, flush, stream):
    """Device time (ms) of `steps` calls of step(), L2 flushed before each."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for k in range(steps):
        flush.zero_()
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b_) for a, b_ in ev)


def measure_mixed(args, eng, b, H, D, dD, dJ, dK, dg, flush, stream, world):
    """The mixed form at MIXED_CUTOFF: FP32 quadrature for quartets whose
    Schwarz x density bound is below it (autotuned split per class), timed like
    the FP64 step, with its energy, Fock and gradient errors against FP64."""
    from iqcp_b200 import FP64, MIXED
    F64 = eng.build_fock(H, D)
    g64 = eng.eri_gradient(D, 1.0)
    e64 = 0.5 * float(np.sum(D * (H + F64)))
    eng.set_precision(MIXED, MIXED_CUTOFF)
    eng.autotune(dD.data_ptr(), 2)

    def step():
        eng.jk_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
        dg.zero_()
        eng.eri_gradient_device(dD.data_ptr(), 1.0, dg.data_ptr())

    for _ in range(args.warmup):
        step()
    t_ms = max_over_ranks(timed_steps(step, args.steps, flush, stream), world)
    eng.jk_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
    nq = eng.last_stats()
    eng.eri_gradient_device(dD.data_ptr(), 1.0, dg.data_ptr())
    ng = eng.last_stats()
    F = eng.build_fock(H, D)
    g = eng.eri_gradient(D, 1.0)
    e = 0.5 * float(np.sum(D * (H + F)))
    modes = eng.kernel_modes()
    eng.set_precision(FP64)
    de, dgmax = abs(e - e64), float(np.abs(g - g64).max())
    return {"cutoff": MIXED_CUTOFF, "value": job_throughput(world, args.steps, t_ms * 1e-3), "unit": UNIT,
            "ms_per_step": t_ms / args.steps,
            "energy_error_ha": de, "fock_max_error_ha": float(np.abs(F - F64).max()),
            "grad_max_error_ha_bohr": dgmax, "within_bounds": bool(de <= 1e-6 and dgmax <= 1e-6),
            "fp32_quartet_share_jk": nq["fp32_quartets"] / max(nq["quartets"], 1),
            "fp32_quartet_share_grad": ng["fp32_quartets"] / max(ng["quartets"], 1),
            "split_classes": {"jk": int(((modes[2] >= 0) & (modes[2] < 4)).sum()),
                              "grad": int(((modes[3] >= 0) & (modes[3] < 4)).sum()), "of": 21},
            "note": "FP32 quadrature (FP64 roots, weights, accumulation) for quartets with "
                    "Q_ij Q_kl max|D| (gradient: max|D|^2) below the cutoff, in the classes where the autotuner "
                    "found the FP64/FP32 split faster than FP64 alone; errors against the FP64 form at the same "
                    "density"}


def measure_batch(args):
    """Batched context: BATCH_SIZE seeded geometries of uneven size through one
    context; one step = one J/K build + one gradient of every geometry."""
    import torch
    from iqcp_b200 import BasisSet
    from iqcp_b200.batch_scf import BatchRHF
    from iqcp_b200.molecules import batch_geometries
    t0 = time.perf_counter()
    geoms = batch_geometries(args.batch, seed=args.seed)
    bases = [BasisSet.build(a, "6-31g*") for a in geoms]
    scf = BatchRHF(bases)          # packed H, core-guess densities, batched context
    eng = scf.eng
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    eng.autotune(scf.D_p.data_ptr(), 1)
    setup_s = time.perf_counter() - t0
    J = torch.empty_like(scf.D_p)
    K = torch.empty_like(scf.D_p)
    g = torch.zeros((eng.n_atoms, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def jk():
        eng.jk_device(scf.D_p.data_ptr(), J.data_ptr(), K.data_ptr())

    def grad():
        g.zero_()
        eng.eri_gradient_device(scf.D_p.data_ptr(), 1.0, g.data_ptr())

    jk()
    grad()
    steps = max(1, min(args.steps, 3))
    tj = timed_steps(jk, steps, flush, stream) / steps
    tg = timed_steps(grad, steps, flush, stream) / steps
    nbf = np.array([bb.n_basis for bb in bases])
    out = {"geometries": args.batch, "basis": "6-31g*", "atoms": [int(min(len(a) for a in geoms)),
                                                                 int(max(len(a) for a in geoms))],
           "nbf_total": int(nbf.sum()), "nbf_range": [int(nbf.min()), int(nbf.max())],
           "jk_ms": tj, "grad_ms": tg, "jk_builds_per_s": args.batch / (tj * 1e-3),
           "grad_evals_per_s": args.batch / (tg * 1e-3),
           "geometry_steps_per_s": args.batch / ((tj + tg) * 1e-3), "setup_s": setup_s,
           "density": "core-Hamiltonian guess of each geometry (J/K cost depends on the Schwarz lists, not D)"}
    if args.batch_scf:
        t1 = time.perf_counter()
        res = scf.run(handoff=0.9, handoff_after=10)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        scf.gradients()
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        out["scf"] = {"iterations": res.iterations, "converged": int(res.converged.sum()),
                      "scf_s": t2 - t1, "gradient_s": t3 - t2,
                      "geometries_per_s": args.batch / (t3 - t1),
                      "note": "RHF to dE 1e-9, rms dD 1e-7, DIIS error 1e-5; one CUDA graph per iteration "
                              "(Fock build, DIIS, purification); once 90 % have converged the rest continue "
                              "in a batch of their own; energy + gradient per geometry"}
    scf.eng.close()
    return out


def run_reference(args, rank):
    """Reference arm: the oracle's CPU restatement, bounded samples per step."""
    if rank != 0:
        return
    from iqcp_b200 import BasisSet
    from iqcp_b200.molecules import workload
    import oracle
    atoms, basis = workload(WORKLOAD, args.seed)
    b = BasisSet.build(atoms, basis)
    rng = np.random.default_rng(args.seed)
    A = rng.normal(size=(b.n_basis, b.n_basis)) * 0.05
    D = A + A.T
    stride = max(args.cpu_sample_stride * 4, 1)
    for w in range(args.warmup):
        cpu_baseline(b, D, stride, w % stride)
    times = []
    for k in range(args.steps):
        r = cpu_baseline(b, D, stride, (args.warmup + k) % stride)
        times.append(1.0 / r["value"])
    t = float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": 1.0 / t, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded molecule)",
            "config": workload_config(b, args.seed),
            "cpu_baseline": {"value": 1.0 / t, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port",
                             "sample": "per step: every %d-th bra shell pair (rotating phase), scaled by %d"
                                       % (stride, stride)},
            "e2e": {"value": 1.0 / t, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's Rust path cannot be built here (no cargo); its algorithm restated in "
                    "C++ (oracle/) is timed on all host threads"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from iqcp_b200 import BasisSet, FockEngine, measure_peak
    from iqcp_b200.molecules import workload
    from iqcp_b200.scf import rhf_scf

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    atoms, basis = workload(WORKLOAD, args.seed)
    b = BasisSet.build(atoms, basis)
    n = b.n_basis
    stream = torch.cuda.current_stream()
    eng = FockEngine(b, device=local)
    eng.set_stream(stream.cuda_stream)
    # converged RHF density (set-up, not timed)
    S, T, V = eng.one_electron()
    H = T + V
    scf = rhf_scf(S, H, b.nuclear_repulsion(), b.n_electrons // 2, eng.build_fock, e_tol=1e-8, d_tol=1e-6)
    D = scf.density
    dD = torch.from_numpy(D).to("cuda")
    dJ = torch.empty_like(dD)
    dK = torch.empty_like(dD)
    dg = torch.zeros((b.n_atoms, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(b, D, args.cpu_sample_stride)
    peak64 = measure_peak("fp64")
    peak32 = measure_peak("fp32")

    def step():
        eng.jk_device(dD.data_ptr(), dJ.data_ptr(), dK.data_ptr())
        l1 = eng.kernel_launches()
        p1 = eng.launch_profile()
        dg.zero_()
        eng.eri_gradient_device(dD.data_ptr(), 1.0, dg.data_ptr())
        l2 = eng.kernel_launches()
        p2 = eng.launch_profile()
        return l1 + l2 + 1, p1 + p2

    # kernel variant per class, picked on this density (set-up, not timed)
    if args.modes:
        for item in args.modes.split(","):
            kind, m = item.split(":")
            eng.set_kernel_mode(kind, mode=int(m))
        modes = eng.kernel_modes()
    else:
        modes = eng.autotune(dD.data_ptr(), 2)
    for _ in range(args.warmup):
        step()
    eng.set_profiling(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    per_kernel = {}
    launches = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            nl, prof = step()
            ev[k][1].record(stream)
            launches += nl
            for p in prof:
                key = (p["kind"], p["X"], p["Y"])
                acc = per_kernel.setdefault(key, [0.0, 0, p["cls"], p["quartets"]])
                acc[0] += p["ms"]
                acc[1] += 1
        torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    eng.set_profiling(False)
    t_ms = max_over_ranks(sum(a.elapsed_time(b_) for a, b_ in ev), world)
    if world > 1:
        dist.barrier()
    clocks = clk.summary()
    value = job_throughput(world, args.steps, t_ms * 1e-3)

    # end to end through the public host-buffer API (pinned host memory)
    hD = torch.from_numpy(D).pin_memory().numpy()
    hJ = torch.empty((n, n), dtype=torch.float64).pin_memory().numpy()
    hK = torch.empty((n, n), dtype=torch.float64).pin_memory().numpy()
    e2e_t = 0.0
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, K = eng.build_jk(hD)
        g = eng.eri_gradient(hD, 1.0)
        e2e_t += time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_t, world)
    e2e = {"value": job_throughput(world, args.steps, e2e_t), "unit": UNIT,
           "h2d_bytes_per_step": 2 * n * n * 8 + b.n_atoms * 3 * 8,
           "d2h_bytes_per_step": 2 * n * n * 8 + b.n_atoms * 3 * 8}

    mixed = None if args.no_mixed else measure_mixed(args, eng, b, H, D, dD, dJ, dK, dg, flush, stream, world)
    batch = None
    if world == 1 and args.batch > 0:
        batch = measure_batch(args)

    # roofline of the dominant quartet kernel (FP64 pipe)
    fl_jk, pq_jk, q_jk = eng.model_flops("jk")
    fl_gr, pq_gr, q_gr = eng.model_flops("grad")
    dom = max(per_kernel.items(), key=lambda kv: kv[1][0])
    (kind, X, Y), (tot_ms, cnt, cls, nq) = dom
    avg_ms = tot_ms / cnt
    flops = (fl_jk if kind == "jk" else fl_gr)[X, Y]
    achieved = flops / (avg_ms * 1e-3) * 1e-12
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        traffic = tr.get("%s%s" % (kind, cls))
    except (OSError, ValueError):
        pass
    total_model = float(fl_jk.sum() + fl_gr.sum())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 40-atom molecule, converged RHF density)",
        "config": workload_config(b, args.seed),
        "jk_builds_per_s_fp64": None, "grad_evals_per_s_fp64": None,
        "e2e": e2e,
        "roofline": {"bound": "fp64", "kernel": "%s %s" % (kind, cls), "achieved": achieved, "peak": peak64,
                     "unit": "TFLOP/s", "frac": achieved / peak64, "traffic": traffic,
                     "peak_source": "measured live: DFMA throughput probe (iqcp_measure_peak); "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "flops_model": "closed-form per surviving primitive quartet (host.cu class_cost)",
                     "avg_launch_ms": avg_ms},
        "step_model_tflops": total_model / (t_ms / args.steps * 1e-3) * 1e-12,
        "fp32_peak_tflops": peak32,
        "clocks": clocks, "gpu_launches": launches,
        "kernels": {"%s %s" % (k[0], v[2]): round(v[0] / v[1], 4) for k, v in sorted(per_kernel.items())},
        "scf": {"energy": scf.energy, "iterations": scf.iterations, "converged": bool(scf.converged)},
        "kernel_modes": {"jk": modes[0].tolist(), "grad": modes[1].tolist(),
                         "legend": "rows bra class, cols ket class (ss ps pp ds dp dd); 0 thread/quartet, "
                                   "1 warp/quartet, 2 8 lanes/quartet, 3 32 lanes/quartet"},
    }
    jk_ms = sum(v[0] / v[1] for k, v in per_kernel.items() if k[0] == "jk")
    gr_ms = sum(v[0] / v[1] for k, v in per_kernel.items() if k[0] == "grad")
    line["jk_builds_per_s_fp64"] = 1e3 / jk_ms
    line["grad_evals_per_s_fp64"] = 1e3 / gr_ms
    if mixed is not None:
        line["mixed"] = mixed
    if batch is not None:
        line["batch"] = batch
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
