#!/usr/bin/env python
"""DEER samples/sec on one B200 (or N replicas, one per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one DEER block solved to convergence, tape generation
and per-sample logp included): the anisotropic diagonal Gaussian, D = 100,
precisions log-uniform in [1e-2, 1e2] (seed 1), eps = 0.05, T = 16384,
jacobian = :diag, FP32 state, x0 ~ N(0, I), sampler defaults otherwise.
The path does not shard (one chain), so N GPUs run N independent replicas
(different tape seeds): weak scaling, no data-path collective.

Printed JSON: value = device-timed samples/s with inputs resident in HBM (L2
flushed between steps), e2e = the same through pmcmc.sample() with host
buffers (one call of 8 blocks per step, wall clock; e2e.one_block: one block
per call), plain_gpu = the unfused reference-structured GPU path, roofline of
the sweep kernel, cpu_baseline = the FP64 CPU restatement of the reference
algorithm on this host's cores.

Secondary measurements (not the headline line; 1 GPU):
    python bench.py --workload logistic_n10k_d256    # N=10000, D=256, T=65536, :stoch_diag
    python bench.py --workload corr_gauss_d64_full   # D=64, T=8192, :full
    python bench.py --workload logistic_fleet        # 32 uneven logistic chains (N, T / 4)
--small shrinks T (logistic 4096, correlated Gaussian 1024) for profiler captures.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "parallelmcmc.jl_b200"))

METRIC = "DEER samples/sec, batched+mixed vs plain GPU DEER, at trace err ≤1e-5 vs FP64"
WORKLOAD = "diag_gauss_D100_T16384_diag_f32"
E2E_BLOCKS = 8  # blocks of T samples per end-to-end sample() call
STEP_BLOCKS = 8  # blocks of T samples per timed device-resident sample() call
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
L2_FLUSH_BYTES = 512 << 20


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "100"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, parts[2:]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_block(model, sampler, x0, seed, block, nthreads):
    """The FP64 CPU restatement of the reference algorithm (per-t :diag with D JVPs
    per column, DEER.jl:420-468; Hillis-Steele scan, DEERScan.jl:102-173) on one block."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    tg = model.target
    otg = O.Target.diag_gauss(tg["prec"], tg["mean"])
    Xi, u = O.tape(seed, block, model.dim, sampler.T)
    t0 = time.perf_counter()
    S, info = O.deer_solve(otg, sampler.epsilon, np.asarray(x0, np.float64), Xi, u, seed, block,
                           jacobian=sampler.jacobian, damping=sampler.damping,
                           tol_abs=sampler.tol_abs, tol_rel=sampler.tol_rel,
                           maxiter=sampler.maxiter, probes=sampler.probes, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return S, info, dt


def cpu_sequential_block(model, sampler, x0, seed, block):
    """The sequential taped MALA chain (MALA.jl:322-346, 377-411) on one block, one
    thread, FP64: the trace DEER reproduces."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    tg = model.target
    otg = O.Target.diag_gauss(tg["prec"], tg["mean"])
    Xi, u = O.tape(seed, block, model.dim, sampler.T)
    t0 = time.perf_counter()
    O.mala_sequential(otg, sampler.epsilon, np.asarray(x0, np.float64), Xi, u)
    return time.perf_counter() - t0


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    from pmcmc import configs
    model, sampler, x0, meta = configs.aniso_diag_d100()
    nthreads = os.cpu_count() or 1
    for w in range(args.warmup):
        cpu_reference_block(model, sampler, x0, meta["seed"], w, nthreads)
    times, iters = [], []
    for k in range(args.steps):
        _, info, dt = cpu_reference_block(model, sampler, x0, meta["seed"], args.warmup + k,
                                          nthreads)
        times.append(dt)
        iters.append(info["iters"])
    total = sum(times)
    value = args.steps * sampler.T / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, see config)",
        "config": {"workload": WORKLOAD, "D": 100, "T": sampler.T, "eps": 0.05,
                   "jacobian": "diag", "newton_iters_mean": statistics.mean(iters)},
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": nthreads, "kind": "port",
                         "sample": "full blocks: FP64 C restatement of the reference CPU DEER "
                                   "(per-t :diag with D JVPs per column, doubling scan), OpenMP"},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "Julia is not installed; the reference arm is the oracle port of its algorithm",
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    import pmcmc
    from pmcmc import _lib as L
    from pmcmc import configs

    world, rank, local = dist_setup()
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one explicit stream for the L2 flush, the CUDA events and the library, so that
    # the events bracket the solve (torch's default stream is the legacy stream 0,
    # which a handle would replace by a non-blocking stream of its own)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    h = pmcmc.Handle(local, stream=stream.cuda_stream)
    lib = L.load()

    model, sampler, x0, meta = configs.aniso_diag_d100()
    D, T = model.dim, sampler.T
    seed = meta["seed"] + 7919 * rank  # replicas: each rank its own tape stream
    tgt = model.device_target(h)
    x0_dev = torch.from_numpy(np.asarray(x0)).to(dev)
    S_dev = torch.empty((T, D), dtype=torch.float32, device=dev)
    lp_dev = torch.empty((T,), dtype=torch.float32, device=dev)
    acc_dev = torch.empty((T,), dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def solve_dev(smp, block):
        info = L.Info()
        p = smp.params()
        rc = lib.pmcmc_deer_solve(h.ptr, tgt, C.byref(p), x0_dev.data_ptr(), seed, block,
                                  S_dev.data_ptr(), lp_dev.data_ptr(), acc_dev.data_ptr(),
                                  L.MEM_DEVICE, C.byref(info))
        L.check(rc, h.ptr, "deer_solve")
        return info

    def timed(smp, nsteps, block0):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(nsteps)]
        infos = []
        for k in range(nsteps):
            flush.zero_()  # L2 flush (512 MB > 126 MB L2), outside the timed events
            ev[k][0].record(stream)
            infos.append(solve_dev(smp, block0 + k))
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in ev], infos

    # A step is one sample() call of STEP_BLOCKS blocks into HBM buffers: block b + 1
    # starts from block b's last column on the device, the blocks run back to back.
    S_run = torch.empty((STEP_BLOCKS * T, D), dtype=torch.float32, device=dev)
    lp_run = torch.empty((STEP_BLOCKS * T,), dtype=torch.float32, device=dev)
    acc_run = torch.empty((STEP_BLOCKS * T,), dtype=torch.uint8, device=dev)

    def timed_run(smp, nsteps, seed0):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(nsteps)]
        infos = []
        for k in range(nsteps):
            flush.zero_()
            ev[k][0].record(stream)
            info = L.Info()
            p = smp.params()
            rc = lib.pmcmc_sample(h.ptr, tgt, C.byref(p), x0_dev.data_ptr(), seed0 + k,
                                  STEP_BLOCKS * T, S_run.data_ptr(), lp_run.data_ptr(),
                                  acc_run.data_ptr(), L.MEM_DEVICE, C.byref(info))
            L.check(rc, h.ptr, "sample")
            ev[k][1].record(stream)
            infos.append(info)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in ev], infos

    # ---- warm-up and timed region (device-resident inputs/outputs)
    timed_run(sampler, args.warmup, seed + 100)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ms, infos = timed_run(sampler, args.steps, seed + 1000)
    torch.cuda.synchronize(dev)
    total_ms = sum(ms)
    if pg:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps * STEP_BLOCKS * T / (total_ms / 1e3)
    iters = [i.iters / STEP_BLOCKS for i in infos]  # Newton sweeps a block
    persistent = bool(infos[0].path & 32)
    # one cooperative launch per block (persistent solve), else init + sweeps + finalize
    launches = sum(STEP_BLOCKS * (1 if persistent else 2) + (0 if persistent else i.iters)
                   for i in infos)
    # the same blocks one solve() call each (a host round trip between blocks)
    timed(sampler, 2, 0)
    ms1, _ = timed(sampler, args.steps, 1000)
    value_one_call = world * args.steps * T / (sum(ms1) / 1e3)

    # ---- parity of the timed workload: first timed block vs the FP64 sequential oracle
    parity = {}
    if rank == 0:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            solve_dev(sampler, 1000)
            S = S_dev.cpu().numpy().T.astype(np.float64)
            acc = acc_dev.cpu().numpy().astype(bool)
            Xi, u = O.tape(seed, 1000, D, T)
            otg = O.Target.diag_gauss(model.target["prec"])
            S_seq, acc_seq, _ = O.mala_sequential(otg, sampler.epsilon,
                                                  np.asarray(x0, np.float64), Xi, u)
            err = float(np.max(np.linalg.norm(S - S_seq, axis=0) /
                               np.maximum(np.linalg.norm(S_seq, axis=0), 1e-30)))
            parity = {"trace_err_vs_fp64": err, "accept_identical": bool(np.array_equal(acc, acc_seq)),
                      "accept_rate": float(acc.mean())}
        except Exception as e:  # parity is reported, never fatal for the timing
            parity = {"error": repr(e)}

    # ---- plain GPU DEER (unfused, reference-structured) on the same workload
    plain = pmcmc.ParallelMALASampler(sampler.epsilon, T=T, jacobian=sampler.jacobian,
                                      dtype=np.float32, exec="plain")
    timed_run(plain, 1, seed + 1900)
    pms, pinfos = timed_run(plain, max(3, args.steps // 4), seed + 2000)
    plain_value = len(pms) * STEP_BLOCKS * T / (sum(pms) / 1e3)

    # ---- roofline of the dominant kernel (the fused sweep), CUDA events per launch
    h.set_profiling(True)
    for k in range(max(3, args.steps // 2)):
        flush.zero_()
        solve_dev(sampler, 3000 + k)
    torch.cuda.synchronize(dev)
    prof = h.profile(reset=True)
    h.set_profiling(False)
    sweep_bytes = 12 * D * T + 8 * T  # one Newton sweep (S read, Xi read, S write, u read, logp write)
    hbm, src = peaks()
    if prof["solve_launches"]:
        # persistent kernel: one launch = tape + every sweep + verification of a block
        kernel = "deer_persist_kernel"
        launch_ms = prof["solve_ms"] / prof["solve_launches"]
        sweeps = prof["solve_sweeps"] / prof["solve_launches"]
        alg_bytes = sweeps * sweep_bytes
        min_bytes = 4 * D * T + 5 * T  # S, logp, accept out; S and the tape stay on chip
        nprof = prof["solve_launches"]
        # dram__bytes_read.sum + dram__bytes_write.sum per block, from the ncu capture of
        # an 8-block launch of this workload (136,704 + 1,610,240 B over 8 blocks),
        # summarised in profiles/deer_persist_kernel_aniso_diag_d100.md
        traffic = 218368
    else:
        kernel = "deer_sweep_kernel"
        launch_ms = prof["sweep_ms"] / max(1, prof["sweep_launches"])
        sweeps = 1.0
        alg_bytes = sweep_bytes
        min_bytes = 8 * D * T + 4 * T  # what this kernel must move (tape regenerated in registers)
        nprof = prof["sweep_launches"]
        # dram__bytes_read.sum + dram__bytes_write.sum of one sweep launch of this workload,
        # from the ncu capture summarised in profiles/deer_sweep_kernel_aniso_diag_d100.md
        traffic = 6754048
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9

    # ---- sequential MALA on the device (pmcmc_mala_chains): one chain over the same
    # block, and a chain a warp on every SM for throughput
    def chains_rate(n):
        x0c = x0_dev.repeat(n, 1).contiguous()
        sd = torch.arange(n, dtype=torch.int64, device=dev) + seed
        Sc = torch.empty((n, T, D), dtype=torch.float32, device=dev)
        p = sampler.params()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.check(lib.pmcmc_mala_chains(h.ptr, tgt, C.byref(p), n, x0c.data_ptr(), sd.data_ptr(),
                                      1000, Sc.data_ptr(), None, None, L.MEM_DEVICE), h.ptr,
                "mala_chains")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return n * T / (e0.elapsed_time(e1) / 1e3)

    chains_rate(1)
    seq_one = chains_rate(1)
    seq_many = chains_rate(8 * torch.cuda.get_device_properties(dev).multi_processor_count)

    # ---- end to end through the public API with host buffers: one sample() call of
    # E2E_BLOCKS blocks per step (x0 in, the chain's values, logp and accept flags out;
    # block b's copy-out overlaps block b + 1's solve), and of one block for reference
    x0_host = torch.tensor(np.asarray(x0, np.float32)).pin_memory().numpy()

    def e2e(nblocks, nsteps):
        pmcmc.sample(model, sampler, nblocks * T, seed=seed, initial_params=x0_host, handle=h)
        ts = []
        for k in range(nsteps):
            t0 = time.perf_counter()
            pmcmc.sample(model, sampler, nblocks * T, seed=seed + 1 + k, initial_params=x0_host,
                         handle=h)
            ts.append(time.perf_counter() - t0)
        total = sum(ts)
        if pg:
            t = torch.tensor([total], device=dev, dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            total = float(t.item())
        return world * nsteps * nblocks * T / total

    e2e_val = e2e(E2E_BLOCKS, max(3, args.steps // 2))
    e2e_one = e2e(1, max(3, args.steps // 2))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        _, cinfo, cdt = cpu_reference_block(model, sampler, x0, seed, 0, nthreads)
        cpu = {"value": T / cdt, "unit": "samples/s", "cores": nthreads, "kind": "port",
               "sample": f"one full block (T={T}): FP64 C restatement of the reference CPU DEER "
                         f"(per-t :diag, D JVPs per column, doubling scan), "
                         f"{cinfo['iters']} Newton iterations, OpenMP"}
        sdt = cpu_sequential_block(model, sampler, x0, seed, 0)
        cpu["sequential_mala"] = {"value": T / sdt, "unit": "samples/s", "cores": 1,
                                  "sample": f"the sequential taped MALA chain over the same "
                                            f"block (T={T}), FP64 C, one thread"}

    if pg:
        pg.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 + counter-based Philox tape)",
            "config": {"workload": WORKLOAD, "D": D, "T": T, "eps": 0.05, "jacobian": "diag",
                       "step": f"pmcmc_sample of {STEP_BLOCKS} blocks (N={STEP_BLOCKS}*T) into "
                               f"HBM buffers, x0 in HBM; CUDA events on the launching stream",
                       "one_block_per_call": {"value": value_one_call, "unit": "samples/s",
                                              "step": "pmcmc_deer_solve of one block"},
                       "state": "f32", "logalpha": "f64", "l2": "flushed (512 MB write) "
                       "between timed steps", "parallelism": f"replicas x{world}",
                       "newton_iters_mean": statistics.mean(iters),
                       "path": [n for b, n in L.PATH_BITS if infos[0].path & b]},
            "e2e": {"value": e2e_val, "unit": "samples/s", "h2d_bytes_per_step": 4 * D,
                    "d2h_bytes_per_step": E2E_BLOCKS * (4 * D * T + 4 * T + T),
                    "step": f"pmcmc.sample(N={E2E_BLOCKS}*T) from pinned x0 into pinned host "
                            f"arrays, wall clock",
                    "one_block": {"value": e2e_one, "step": "pmcmc.sample(N=T)",
                                  "d2h_bytes_per_step": 4 * D * T + 4 * T + T}},
            "gpu_sequential_mala": {"one_chain": seq_one,
                                    "one_chain_speedup_of_deer": value / world / seq_one,
                                    "chains_8_per_sm": seq_many, "unit": "samples/s",
                                    "note": "independent taped MALA chains, one warp each "
                                            "(pmcmc_mala_chains), same block and tape"},
            "plain_gpu": {"value": plain_value, "unit": "samples/s",
                          "newton_iters_mean": statistics.mean(i.iters / STEP_BLOCKS for i in pinfos),
                          "speedup_fused_over_plain": value / world / plain_value},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_source": src,
                         "kernel": kernel, "avg_launch_ms": launch_ms,
                         "sweeps_per_launch": sweeps,
                         "alg_bytes_per_launch": alg_bytes,
                         "kernel_min_bytes_per_launch": min_bytes,
                         "launches_profiled": nprof},
            "cpu_baseline": cpu,
            "parity": parity,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def run_secondary(args):
    """Logistic regression (tensor-core contraction passes) or the correlated
    Gaussian in :full mode: device-timed solves, Newton iterations, accept
    rate, and the roofline of the dominant kernel."""
    import ctypes as C

    import numpy as np
    import torch

    import pmcmc
    from pmcmc import _lib as L
    from pmcmc import configs

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)  # flush, events and library in one stream
    torch.cuda.set_stream(stream)
    h = pmcmc.Handle(0, stream=stream.cuda_stream)
    lib = L.load()
    logistic = args.workload == "logistic_n10k_d256"
    if logistic:
        model, sampler, x0, meta = configs.logistic_n10k_d256(T=4096 if args.small else 65536,
                                                              D=args.dim)
    else:
        model, sampler, x0, meta = configs.correlated_gauss_d64(T=1024 if args.small else 8192)
        # the sampler's default stopping rule (1e-6 + 1e-5 |S|) allows ~1e-5 relative
        # error in itself; the 1e-5 trace-error bar needs a tighter one
        sampler.tol_abs, sampler.tol_rel = 1e-7, 1e-6
    D, T = model.dim, sampler.T
    tgt = model.device_target(h)
    x0_dev = torch.from_numpy(np.asarray(x0, np.float32)).to(dev)
    S_dev = torch.empty((T, D), dtype=torch.float32, device=dev)
    lp_dev = torch.empty((T,), dtype=torch.float32, device=dev)
    acc_dev = torch.empty((T,), dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def solve_dev(smp, block):
        info = L.Info()
        p = smp.params()
        rc = lib.pmcmc_deer_solve(h.ptr, tgt, C.byref(p), x0_dev.data_ptr(), meta["seed"], block,
                                  S_dev.data_ptr(), lp_dev.data_ptr(), acc_dev.data_ptr(),
                                  L.MEM_DEVICE, C.byref(info))
        L.check(rc, h.ptr, "deer_solve")
        return info

    for w in range(args.warmup):
        solve_dev(sampler, w)
    torch.cuda.synchronize(dev)
    ms, infos = [], []
    with ClockSampler(0) as clk:
        for k in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            infos.append(solve_dev(sampler, 1000 + k))
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
    value = args.steps * T / (sum(ms) / 1e3)
    iters = statistics.mean(i.iters for i in infos)
    acc_rate = statistics.mean(i.n_accept / T for i in infos)

    h.set_profiling(True)
    solve_dev(sampler, 3000)
    torch.cuda.synchronize(dev)
    prof = h.profile(reset=True)
    h.set_profiling(False)
    hbm, src = peaks()
    line = {"metric": METRIC, "secondary": True, "value": value, "unit": "samples/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sum(ms) / args.steps, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 + counter-based Philox tape)",
            "config": {"workload": meta["workload"], "D": D, "T": T, "eps": sampler.epsilon,
                       "jacobian": sampler.jacobian, "tol_abs": sampler.tol_abs,
                       "tol_rel": sampler.tol_rel, "newton_iters_mean": iters,
                       "accept_rate": acc_rate, "path": infos[-1].as_dict()["path_names"]},
            "clocks": clk.summary()}
    if logistic:
        # plain FP32 GPU DEER on the first timed block: unfused kernels, cuBLAS FP32
        # contractions, the convergence test on the host after every iteration
        import dataclasses
        plain = dataclasses.replace(sampler, exec="plain")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        pinfo = solve_dev(plain, 1000)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        pms = e0.elapsed_time(e1)
        line["plain_gpu"] = {"value": T / (pms / 1e3), "unit": "samples/s", "block": 1000,
                             "newton_iters": pinfo.iters, "converged": bool(pinfo.converged),
                             "fused_newton_iters_same_block": infos[0].iters,
                             "speedup_fused_over_plain": value / (T / (pms / 1e3))}
        N = meta.get("N_rows", 10_000)
        pass_ms = prof["pass_ms"] / max(1, prof["pass_launches"])
        flops = 8.0 * N * D * T  # two GEMMs of 2 N D (2T) per contraction pass
        try:
            with open(PEAKS_PATH) as f:
                tpk, tsrc = float(json.load(f)["bf16_tflops"]), "measured (bf16 dense, burst)"
        except Exception:
            tpk, tsrc = 1590.0, "fallback"
        achieved = flops / (pass_ms / 1e3) / 1e12
        kname = "logistic_pass_tc_wide_kernel" if D > 256 else "logistic_pass_tc_kernel"
        line["roofline"] = {"bound": "tensor", "kernel": f"{kname} (+ mid kernel)",
                            "achieved": achieved, "peak": tpk, "unit": "TFLOP/s",
                            "frac": achieved / tpk, "peak_source": tsrc,
                            "avg_launch_ms": pass_ms, "alg_flops_per_launch": flops,
                            "executed_mma_flops_per_launch": 2 * flops,
                            "sweep_ms": prof["sweep_ms"] / max(1, prof["sweep_launches"])}
    else:
        sweep_ms = prof["sweep_ms"] / max(1, prof["sweep_launches"])
        Dq = 64
        # eval: S' and xi' read, u', v', r' written; chunk and apply: u', v', r' read;
        # apply: S and S' read and written; log u and accept flags
        alg_bytes = 4 * T * (13 * Dq + 2 * D) + 9 * T
        achieved = alg_bytes / (sweep_ms / 1e3) / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": "full sweep (eval+chunk+carry+apply)",
                            "achieved": achieved, "peak": hbm, "unit": "GB/s",
                            "frac": achieved / hbm, "peak_source": src, "avg_sweep_ms": sweep_ms,
                            "alg_bytes_per_sweep": alg_bytes,
                            "note": "latency-bound: the chunk, carry and replay recursions are sequential"}
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        solve_dev(sampler, 1000)
        S = S_dev.cpu().numpy().T.astype(np.float64)
        acc = acc_dev.cpu().numpy().astype(bool)
        Xi, u = O.tape(meta["seed"], 1000, D, T)
        S_seq, acc_seq, _ = O.mala_sequential(O.Target.dense_gauss(model.target["prec"]),
                                              sampler.epsilon, np.asarray(x0, np.float64), Xi, u)
        line["parity"] = {"trace_err_vs_fp64": float(np.max(
            np.linalg.norm(S - S_seq, axis=0) / np.maximum(np.linalg.norm(S_seq, axis=0), 1e-30))),
            "accept_identical": bool(np.array_equal(acc, acc_seq))}
    print(json.dumps(line), flush=True)


def run_fleet(args):
    """A bounded sample of the uneven logistic fleet (chains 0..n-1 of the
    512-chain configuration, N and T scaled by 1/4): all chains through
    pmcmc_fleet_solve on 8 worker streams, and the same chains one at a time."""
    import numpy as np
    import torch

    import pmcmc
    from pmcmc import configs

    n = 8 if args.small else 32
    chains = configs.logistic_fleet(n_chains=n, scale=0.25)
    h = pmcmc.Handle(0)
    total_T = sum(s.T for _, s, *_ in chains)
    # stiff chains (small D, large N: eps * lambda_max > 2) can diverge in DEER itself,
    # as the FP64 CPU restatement does on them; their status is reported per chain
    pmcmc.fleet_solve(chains, workers=8, handle=h, errors="report")  # warm-up
    times = []
    with ClockSampler(0) as clk:
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = pmcmc.fleet_solve(chains, workers=8, handle=h, errors="report")
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    pmcmc.fleet_solve(chains, workers=1, handle=h, errors="report")
    torch.cuda.synchronize()
    serial = time.perf_counter() - t0
    # plain per-chain FP32 GPU DEER (unfused kernels, cuBLAS FP32 contractions, host
    # convergence test every iteration), the same chains one at a time, one run
    import dataclasses
    plain_chains = [(m, dataclasses.replace(smp, exec="plain"), *rest)
                    for m, smp, *rest in chains]
    t0 = time.perf_counter()
    pres = pmcmc.fleet_solve(plain_chains, workers=1, handle=h, errors="report")
    torch.cuda.synchronize()
    plain_t = time.perf_counter() - t0
    acc = [float(np.mean(r[3])) for r in res]
    iters = [r[1]["iters"] for r in res]
    best = min(times)
    line = {"metric": METRIC, "secondary": True, "value": total_T / best, "unit": "samples/s",
            "n_gpus": 1, "steps": len(times), "warmup": 1, "ms_per_step": 1e3 * best,
            "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 per chain + counter-based Philox tape)",
            "timing": "host wall clock around pmcmc_fleet_solve with device synchronisation "
                      "(chains run on 8 streams); best of the timed runs",
            "config": {"workload": f"logistic_fleet_{n}chains_scale0.25", "chains": n,
                       "D_range": [min(m.dim for m, *_ in chains), max(m.dim for m, *_ in chains)],
                       "N_range": [min(m.target["X"].shape[0] for m, *_ in chains),
                                   max(m.target["X"].shape[0] for m, *_ in chains)],
                       "T_total": total_T, "workers": 8,
                       "newton_iters": {"min": min(iters), "median": statistics.median(iters),
                                        "max": max(iters)},
                       "accept_rate": {"min": min(acc), "median": statistics.median(acc),
                                       "max": max(acc)},
                       "converged": sum(r[1]["converged"] for r in res),
                       "not_converged": sum(1 for r in res
                                            if not r[1]["converged"] and r[1]["status"] == 0),
                       "nonfinite": [i for i, r in enumerate(res) if r[1]["status"] == 4]},
            "one_chain_at_a_time": {"value": total_T / serial, "unit": "samples/s",
                                    "speedup_fleet": serial / best},
            "plain_gpu_per_chain": {"value": total_T / plain_t, "unit": "samples/s",
                                    "speedup_fleet_over_plain": plain_t / best,
                                    "converged": sum(r[1]["converged"] for r in pres),
                                    "newton_iters_median": statistics.median(
                                        r[1]["iters"] for r in pres)},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--workload", default="aniso_diag_d100",
                    choices=["aniso_diag_d100", "logistic_n10k_d256", "corr_gauss_d64_full",
                             "logistic_fleet"])
    ap.add_argument("--dim", type=int, default=256,
                    help="logistic workload: dimension D (256 < D <= 512 runs the wide "
                         "tensor-core pass)")
    ap.add_argument("--small", action="store_true",
                    help="secondary workloads: shorter T for profiler captures")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "logistic_fleet" and args.impl == "ours":
        run_fleet(args)
    elif args.workload != "aniso_diag_d100" and args.impl == "ours":
        run_secondary(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
