#!/usr/bin/env python
"""DEER samples/sec on one B200 (or N replicas, one per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (the metric's batched + mixed-precision configuration):
Bayesian logistic regression, N = 10000 rows, D = 256, X iid N(0,1)/sqrt(D),
theta* ~ N(0, I), y ~ Bernoulli(sigmoid(X theta*)), prior N(0, I), all from
seed 2; eps = 0.01, T = 65536, :stoch_diag with one probe, FP32 state.  One
step is one block of T samples solved to convergence: tape generation, every
Newton sweep (two tensor-core contraction passes, the FP64 decisions of
near-tie columns, the fused finish + scan), the verification pass at the
returned trajectory and the per-sample logp.  The stopping rule is
1e-7 + 1e-6 max|S|: the sampler's default (1e-6 + 1e-5 max|S|) bounds the last
step, and leaves the iterate about 1.2e-5 from the fixed point, above the
metric's 1e-5 trace-error bar.  A block that stops unconverged or non-finite
fails the run.  The path does not shard (one chain), so N GPUs run N
independent replicas (different tape seeds): weak scaling, no collective on
the data path.

Printed JSON: value = device-timed samples/s with the data resident in HBM
(L2 flushed between steps); e2e = the same through pmcmc.sample() with host
buffers; plain_gpu = the reference-structured GPU path (unfused kernels, cuBLAS
FP32 contractions, host convergence test) on the same blocks; parity = a timed
block against the FP64 sequential chain; roofline of the tensor-core pass;
cpu_baseline = the FP64 restatement of the reference's CPU DEER on this host.

Secondary measurements (1 GPU):
    python bench.py --workload aniso_diag_d100       # D=100, T=16384, :diag (persistent kernel)
    python bench.py --workload corr_gauss_d64_full   # D=64, T=8192, :full
    python bench.py --workload logistic_fleet        # 32 uneven logistic chains (N, T / 4)
    python bench.py --workload logistic_fleet_full   # all 512 chains at full N and T
    python bench.py --workload logistic_adjoint      # the logistic adjoint at a solved block
    python bench.py --workload logistic_n10k_d256 --dim 512   # the wide tensor-core pass
--small shrinks T (logistic 4096, correlated Gaussian 1024) for profiler captures.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "parallelmcmc.jl_b200"))

METRIC = "DEER samples/sec, batched+mixed vs plain GPU DEER, at trace err ≤1e-5 vs FP64"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per launch of the profiled kernels, from ncu captures (kernel, workload, bytes)
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "dram_traffic.txt")
L2_FLUSH_BYTES = 512 << 20
TOL = (1e-7, 1e-6)   # headline stopping rule (tol_abs, tol_rel)
REF_T = 128          # reference arm: columns of each complete CPU solve
CPU_T = 256          # cpu_baseline of our arm: columns of the CPU solve


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
            "fallback"


def traffic_of(kernel: str, workload: str):
    """DRAM bytes a launch of `kernel` on `workload` moved in an ncu capture, or None."""
    try:
        with open(TRAFFIC_PATH) as f:
            for ln in f:
                p = ln.split()
                if len(p) >= 3 and not ln.startswith("#") and p[0] == kernel and p[1] == workload:
                    return int(p[2])
    except OSError:
        pass
    return None


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


def headline(T=65536):
    from pmcmc import configs
    model, sampler, x0, meta = configs.logistic_n10k_d256(T=T)
    sampler = dataclasses.replace(sampler, tol_abs=TOL[0], tol_rel=TOL[1])
    return model, sampler, x0, meta


def workload_name(T=65536):
    return f"logistic_N10000_D256_T{T}_stoch_diag_f32"


def trace_err(S, R):
    import numpy as np
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


# --------------------------------------------------------------------------- CPU legs
def cpu_deer_solve(model, sampler, seed, block, T):
    """One complete solve of a T-column block by the FP64 NumPy restatement of the
    reference's CPU DEER on the batched :stoch_diag branch (twelve BLAS GEMMs a
    sweep, MALA.jl:556-628 with bayes_logreg.jl:91-206; doubling scan,
    DEERScan.jl:102-173), BLAS on every host thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import np_oracle as NP
    import oracle as O
    tg = model.target
    D = model.dim
    m = NP.logistic_batched_model(tg["X"], tg["y"], tg["prior_prec"])
    Xi, u = O.tape(seed, block, D, T)
    t0 = time.perf_counter()
    _, info = NP.deer_solve_batched(m, sampler.epsilon, np.zeros(D), np.asarray(Xi, np.float64),
                                    u, lambda it: O.probe(seed, block, it, 0, D, T),
                                    tol_abs=sampler.tol_abs, tol_rel=sampler.tol_rel,
                                    maxiter=sampler.maxiter, damping=sampler.damping)
    return info, time.perf_counter() - t0


def blas_threads():
    try:
        import threadpoolctl
        return max(i.get("num_threads", 1) for i in threadpoolctl.threadpool_info()
                   if i.get("user_api") == "blas")
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    model, sampler, x0, meta = headline()
    for w in range(args.warmup):
        cpu_deer_solve(model, sampler, meta["seed"], w, REF_T)
    times, iters = [], []
    for k in range(args.steps):
        info, dt = cpu_deer_solve(model, sampler, meta["seed"], args.warmup + k, REF_T)
        if not info["converged"]:
            raise SystemExit(f"reference CPU DEER: block {args.warmup + k} not converged: {info}")
        times.append(dt)
        iters.append(info["iters"])
    total = sum(times)
    value = args.steps * REF_T / total
    nth = blas_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, see config)",
        "config": {"workload": workload_name(), "N": 10000, "D": 256, "T": 65536, "eps": 0.01,
                   "jacobian": "stoch_diag", "tol_abs": TOL[0], "tol_rel": TOL[1],
                   "sample": f"each step one complete solve of a {REF_T}-column block of this "
                             f"target (a 65536-column block takes about 55 sweeps of ~2 min "
                             f"each on the CPU; sweeps a solve grow with T, so this rate is "
                             f"an upper bound for full blocks)",
                   "newton_iters_mean": statistics.mean(iters)},
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": nth, "kind": "port",
                         "sample": f"complete {REF_T}-column solves: FP64 NumPy restatement of "
                                   f"the reference's batched CPU DEER (12 BLAS GEMMs a sweep, "
                                   f"single-threaded elementwise work as Julia broadcasts)"},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "Julia is not installed on the GPU box; the reference arm is the oracle port "
                "of its algorithm",
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- our arm
def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    import pmcmc
    from pmcmc import _lib as L

    world, rank, local = dist_setup()
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one explicit stream for the L2 flush, the CUDA events and the library
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    h = pmcmc.Handle(local, stream=stream.cuda_stream)
    lib = L.load()

    model, sampler, x0, meta = headline()
    D, T, N = model.dim, sampler.T, model.target["X"].shape[0]
    seed = meta["seed"] + 7919 * rank  # replicas: each rank its own tape stream
    tgt = model.device_target(h)
    x0_dev = torch.from_numpy(np.asarray(x0, np.float32)).to(dev)
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

    def timed(smp, blocks):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in blocks]
        infos = []
        for k, b in enumerate(blocks):
            flush.zero_()  # L2 flush (512 MB > 126 MB L2), outside the timed events
            ev[k][0].record(stream)
            infos.append(solve_dev(smp, b))
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in ev], infos

    def check_converged(infos, blocks, what):
        for b, i in zip(blocks, infos):
            if not i.converged or i.status:
                line = {"metric": METRIC, "value": None, "unit": "samples/s",
                        "error": f"{what}: block {b} not converged (iters {i.iters}, metric "
                                 f"{i.metric:.3g}, status {i.status}); unconverged blocks are "
                                 f"not samples"}
                print(json.dumps(line), flush=True)
                raise SystemExit(1)

    # ---- warm-up and timed region (data and outputs in HBM)
    timed(sampler, [100 + w for w in range(args.warmup)])
    blocks = [1000 + k for k in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ms, infos = timed(sampler, blocks)
    torch.cuda.synchronize(dev)
    check_converged(infos, blocks, "timed")
    total_ms = sum(ms)
    if pg:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps * T / (total_ms / 1e3)
    iters = [i.iters for i in infos]
    # kernels of ours a block: init; a sweep = 2 passes x (operand split, tensor-core
    # pass, mid) + near-tie selection (margin, select, gather, 2 x loglik, propose,
    # final) + the finish-and-scan sweep kernel; the verification the same without the
    # sweep kernel plus the verify kernel; the logp pass (split, tensor-core pass);
    # finalize.  cuBLAS DGEMMs of the near-tie columns are not counted.
    per_sweep = 6 + 7 + 1
    launches = sum(1 + per_sweep * i.iters + (6 + 7 + 1) + 2 + 1 for i in infos)

    # ---- end to end through the public API with host buffers: pmcmc.sample of one
    # block per step (x0 from pinned memory in, the chain's values, logp and accept
    # flags out to host memory), wall clock
    x0_host = torch.tensor(np.asarray(x0, np.float32)).pin_memory().numpy()

    def e2e(nsteps):
        pmcmc.sample(model, sampler, T, seed=seed + 1, initial_params=x0_host, handle=h)
        ts, oks = [], True
        for k in range(nsteps):
            t0 = time.perf_counter()
            ch = pmcmc.sample(model, sampler, T, seed=seed + 2 + k, initial_params=x0_host,
                              handle=h)
            ts.append(time.perf_counter() - t0)
            oks &= bool(ch.info["converged"])
        total = sum(ts)
        if pg:
            t = torch.tensor([total], device=dev, dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            total = float(t.item())
        return world * nsteps * T / total, oks

    e2e_val, e2e_ok = e2e(max(3, args.steps // 4))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return

    # ---- parity of a timed block: block 1000 solved again (solves repeat bit for bit)
    # against the FP64 sequential chain on the same tape
    parity = {}
    try:
        if args.no_parity:
            raise RuntimeError("skipped (--no-parity)")
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        pinfo = solve_dev(sampler, blocks[0])
        S = S_dev.cpu().numpy().T.astype(np.float64)
        acc = acc_dev.cpu().numpy().astype(bool)
        Xi, u = O.tape(seed, blocks[0], D, T)
        otg = O.Target.logistic(model.target["X"], model.target["y"])
        t0 = time.perf_counter()
        S_seq, acc_seq, la_seq = O.mala_sequential_logistic(otg, sampler.epsilon,
                                                            np.zeros(D), Xi, u)
        seq_s = time.perf_counter() - t0
        m_seq = la_seq - np.log(u.astype(np.float64))
        parity = {"block": blocks[0], "trace_err_vs_fp64": trace_err(S, S_seq),
                  "accept_identical": bool(np.array_equal(acc, acc_seq)),
                  "accept_mismatches": int(np.sum(acc != acc_seq)),
                  "accept_rate": float(acc.mean()), "newton_iters": pinfo.iters,
                  "min_margin_fp64_chain": float(np.abs(m_seq).min()),
                  "min_margin_returned": pinfo.min_margin, "max_defect": pinfo.max_defect,
                  "fp64_chain": f"oracle sequential chain, {os.cpu_count()} threads, "
                                f"{seq_s:.1f} s"}
    except Exception as e:  # parity is reported, never fatal for the timing
        parity = {"error": repr(e)}

    # ---- plain GPU DEER (reference structure: unfused kernels, cuBLAS FP32
    # contractions in pedantic mode, host convergence test every sweep) on the first
    # two timed blocks
    plain = dataclasses.replace(sampler, exec="plain")
    pblocks = blocks[:2]
    pms, pinfos = timed(plain, pblocks)
    p_ok = all(i.converged and not i.status for i in pinfos)
    plain_value = len(pms) * T / (sum(pms) / 1e3)
    same = [ms[k] for k in range(len(pblocks))]
    plain_gpu = {"value": plain_value, "unit": "samples/s", "blocks": pblocks,
                 "newton_iters": [i.iters for i in pinfos], "converged": p_ok,
                 "fused_newton_iters_same_blocks": iters[:len(pblocks)],
                 "speedup_fused_over_plain": (sum(pms) / sum(same)) if p_ok else None,
                 "note": "both paths converged on these blocks" if p_ok else
                         "plain path did not converge: no speed-up reported"}

    # ---- roofline of the dominant kernel: the tensor-core contraction pass, timed
    # with CUDA events around every pass (profiling mode) over one block
    pk, src = peaks()
    h.set_profiling(True)
    flush.zero_()
    solve_dev(sampler, 3000)
    torch.cuda.synchronize(dev)
    prof = h.profile(reset=True)
    h.set_profiling(False)
    pass_ms = prof["pass_ms"] / max(1, prof["pass_launches"])
    flops = 8.0 * N * D * T  # two GEMMs of 2 N D (2T) per contraction pass
    tpk = float(pk.get("bf16_tflops_sustained", pk["bf16_tflops"]))
    achieved = flops / (pass_ms / 1e3) / 1e12
    kname = "logistic_pass_tc_kernel"
    roofline = {"bound": "tensor", "kernel": kname, "achieved": achieved, "peak": tpk,
                "unit": "TFLOP/s", "frac": achieved / tpk, "traffic": traffic_of(kname, workload_name()),
                "peak_source": f"{src}: bf16 dense, sustained (the pass runs inside a "
                               f"seconds-long solve)",
                "avg_launch_ms": pass_ms, "launches_timed": prof["pass_launches"],
                "alg_flops_per_launch": flops,
                "alg_flops_note": "16 N D T a sweep over its two passes (section 8d); value "
                                  "columns run three products (hi*hi, lo*hi, hi*lo) and "
                                  "tangents one, so the tensor pipe executes ~2x",
                "sweep_kernel_ms": prof["sweep_ms"] / max(1, prof["sweep_launches"])}

    # ---- CPU baselines (bounded samples on this host's cores)
    cpu = None
    if world == 1 and not args.no_cpu:
        cinfo, cdt = cpu_deer_solve(model, sampler, seed, 0, CPU_T)
        cpu = {"value": CPU_T / cdt, "unit": "samples/s", "cores": blas_threads(),
               "kind": "port",
               "sample": f"one complete solve of a {CPU_T}-column block of this target "
                         f"({cinfo['iters']} sweeps, {cdt:.1f} s): FP64 NumPy restatement of "
                         f"the reference's batched CPU DEER, 12 BLAS GEMMs a sweep; full "
                         f"65536-column blocks need more sweeps, so this rate is an upper bound"}
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        Ts = 4096
        Xi, u = O.tape(seed, 0, D, Ts)
        otg = O.Target.logistic(model.target["X"], model.target["y"])
        t0 = time.perf_counter()
        O.mala_sequential_logistic(otg, sampler.epsilon, np.zeros(D), Xi, u)
        sdt = time.perf_counter() - t0
        cpu["sequential_mala"] = {"value": Ts / sdt, "unit": "samples/s",
                                  "cores": os.cpu_count(),
                                  "sample": f"the sequential FP64 MALA chain over {Ts} steps "
                                            f"of the same target (oracle C, threaded sums)"}

    secondary = {}
    if not args.no_secondary:
        try:
            secondary["aniso_diag_d100"] = gauss_secondary(h, lib, stream, dev, flush)
        except Exception as e:
            secondary["aniso_diag_d100"] = {"error": repr(e)}

    line = {
        "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded NumPy PCG64 data + counter-based Philox tape)",
        "config": {"workload": workload_name(), "N": N, "D": D, "T": T,
                   "eps": sampler.epsilon, "jacobian": "stoch_diag", "probes": 1,
                   "tol_abs": TOL[0], "tol_rel": TOL[1],
                   "step": "pmcmc_deer_solve of one block, data and outputs in HBM; CUDA "
                           "events on the launching stream",
                   "precision": "FP32 state; contractions on tcgen05 tensor cores with FP16 "
                                "hi/lo split operands (~22 bits) and FP32 accumulation; "
                                "log alpha and Newton metric in FP64; near-tie columns "
                                "decided from an FP64 log alpha",
                   "l2": "flushed (512 MB write) between timed steps",
                   "parallelism": f"replicas x{world}",
                   "newton_iters_mean": statistics.mean(iters),
                   "newton_iters": [min(iters), max(iters)],
                   "accept_rate": statistics.mean(i.n_accept / T for i in infos),
                   "path": [n for b, n in L.PATH_BITS if infos[0].path & b]},
        "e2e": {"value": e2e_val, "unit": "samples/s", "h2d_bytes_per_step": 4 * D,
                "d2h_bytes_per_step": 4 * D * T + 4 * T + T, "converged": e2e_ok,
                "step": "pmcmc.sample(N=T) from a pinned x0 into host arrays (values, logp, "
                        "accept flags), wall clock"},
        "plain_gpu": plain_gpu,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "parity": parity,
        "secondary": secondary,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def gauss_secondary(h, lib, stream, dev, flush):
    """The D = 100 anisotropic diagonal Gaussian (T = 16384, :diag) on the persistent
    kernel: 8-block sample() calls into HBM, the same on the plain path, and a chain
    that moves (eps = 0.005, several sweeps a block)."""
    import ctypes as C

    import numpy as np
    import torch

    from pmcmc import _lib as L
    from pmcmc import configs
    model, sampler, x0, meta = configs.aniso_diag_d100()
    D, T, nb = model.dim, sampler.T, 8
    tgt = model.device_target(h)
    x0_dev = torch.from_numpy(np.asarray(x0)).to(dev)
    S = torch.empty((nb * T, D), dtype=torch.float32, device=dev)
    lp = torch.empty((nb * T,), dtype=torch.float32, device=dev)
    acc = torch.empty((nb * T,), dtype=torch.uint8, device=dev)

    def run(smp, seeds):
        out = []
        for s in seeds:
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info = L.Info()
            p = smp.params()
            L.check(lib.pmcmc_sample(h.ptr, tgt, C.byref(p), x0_dev.data_ptr(), s, nb * T,
                                     S.data_ptr(), lp.data_ptr(), acc.data_ptr(), L.MEM_DEVICE,
                                     C.byref(info)), h.ptr, "sample")
            e1.record(stream)
            torch.cuda.synchronize(dev)
            out.append((e0.elapsed_time(e1), info))
        return out

    res = {}
    for name, smp in (("default", sampler),
                      ("moving_eps0.005", dataclasses.replace(sampler, epsilon=0.005)),
                      ("plain", dataclasses.replace(sampler, exec="plain"))):
        run(smp, [meta["seed"] + 100 + i for i in range(2)])
        r = run(smp, [meta["seed"] + 1000 + i for i in range(5)])
        tot = sum(m for m, _ in r)
        res[name] = {"value": 5 * nb * T / (tot / 1e3), "unit": "samples/s",
                     "sweeps_per_block": statistics.mean(i.iters / nb for _, i in r),
                     "accept_rate": statistics.mean(i.n_accept / (nb * T) for _, i in r),
                     "converged": all(i.converged for _, i in r),
                     "us_per_block": 1e3 * tot / (5 * nb)}
    res["workload"] = meta["workload"]
    res["step"] = f"pmcmc_sample of {nb} blocks into HBM (one persistent launch on the fused path)"
    return res


# --------------------------------------------------------------------------- secondary workloads
def run_secondary(args):
    """Logistic regression at another D or T, or the correlated Gaussian in :full
    mode: device-timed solves, Newton iterations, accept rate, and the roofline of
    the dominant kernel."""
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
        sampler = dataclasses.replace(sampler, tol_abs=TOL[0], tol_rel=TOL[1])
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
    pk, src = peaks()
    line = {"metric": METRIC, "secondary": True, "value": value, "unit": "samples/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sum(ms) / args.steps, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 + counter-based Philox tape)",
            "config": {"workload": meta["workload"], "D": D, "T": T, "eps": sampler.epsilon,
                       "jacobian": sampler.jacobian, "tol_abs": sampler.tol_abs,
                       "tol_rel": sampler.tol_rel, "newton_iters_mean": iters,
                       "accept_rate": acc_rate,
                       "converged": all(i.converged for i in infos),
                       "path": infos[-1].as_dict()["path_names"]},
            "clocks": clk.summary()}
    if logistic:
        N = meta.get("N_rows", 10_000)
        pass_ms = prof["pass_ms"] / max(1, prof["pass_launches"])
        flops = 8.0 * N * D * T  # two GEMMs of 2 N D (2T) per contraction pass
        tpk = float(pk.get("bf16_tflops_sustained", pk["bf16_tflops"]))
        achieved = flops / (pass_ms / 1e3) / 1e12
        kname = "logistic_pass_tc_wide_kernel" if D > 256 else "logistic_pass_tc_kernel"
        line["roofline"] = {"bound": "tensor", "kernel": f"{kname} (+ mid kernel)",
                            "achieved": achieved, "peak": tpk, "unit": "TFLOP/s",
                            "frac": achieved / tpk, "peak_source": f"{src}, sustained",
                            "avg_launch_ms": pass_ms, "alg_flops_per_launch": flops,
                            "sweep_ms": prof["sweep_ms"] / max(1, prof["sweep_launches"])}
    else:
        sweep_ms = prof["sweep_ms"] / max(1, prof["sweep_launches"])
        Dq = 64
        # eval: S' and xi' read, u', v', r' written; chunk and apply: u', v', r' read;
        # apply: S and S' read and written; log u and accept flags
        alg_bytes = 4 * T * (13 * Dq + 2 * D) + 9 * T
        achieved = alg_bytes / (sweep_ms / 1e3) / 1e9
        hbm = float(pk["hbm_gbs"])
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
        line["parity"] = {"trace_err_vs_fp64": trace_err(S, S_seq),
                          "accept_identical": bool(np.array_equal(acc, acc_seq))}
    print(json.dumps(line), flush=True)


def run_gauss(args):
    """The D = 100 diagonal-Gaussian workload alone (persistent kernel)."""
    import torch

    import pmcmc
    from pmcmc import _lib as L
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    h = pmcmc.Handle(0, stream=stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    with ClockSampler(0) as clk:
        res = gauss_secondary(h, L.load(), stream, dev, flush)
    res.update({"metric": METRIC, "secondary": True, "clocks": clk.summary()})
    print(json.dumps(res), flush=True)


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
    if dist_setup()[0] > 1:
        return run_fleet_ranks(args, chains, f"logistic_fleet_{n}chains_scale0.25")
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


def run_adjoint(args):
    """The logistic adjoint at the headline workload: one block solved on the
    tensor cores, then d ESJD / d epsilon and d mean|x|^2 / d epsilon at the
    returned trajectory (FP64 HVP GEMMs and Jacobi iterations), host wall clock
    with device synchronisation."""
    import numpy as np
    import torch

    import pmcmc

    T = 4096 if args.small else 65536
    model, sampler, x0, meta = headline(T=T)
    h = pmcmc.Handle(0)
    dev = torch.device("cuda", 0)
    S, info = pmcmc.solve(model, sampler, x0, seed=meta["seed"] + 1000, block=1000, handle=h)
    if not info["converged"]:
        raise RuntimeError("the block did not converge")
    out = {}
    with ClockSampler(0) as clk:
        for obj in ("esjd", "mean_sq"):
            times = []
            for _ in range(2):
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                g = pmcmc.adjoint(model, sampler, x0, S, objective=obj,
                                  seed=meta["seed"] + 1000, block=1000, handle=h)
                torch.cuda.synchronize(dev)
                times.append(time.perf_counter() - t0)
            out[obj] = {"d_epsilon": g["d_epsilon"], "ms": 1e3 * min(times)}
    line = {"metric": "logistic adjoint d objective / d epsilon at a solved block",
            "secondary": True, "value": out["esjd"]["ms"], "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64 (adjoint), f32 (state)",
            "config": {"workload": workload_name(T), "newton_iters": info["iters"]},
            "objectives": out, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_fleet_ranks(args, chains, workload):
    """The fleet on N GPUs, one process each: every rank solves the chains the
    cost-balanced partition gives it (pmcmc.distributed.fleet_solve_distributed,
    no collective while they solve); the time is the slowest rank's."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import pmcmc
    from pmcmc import distributed as Dd

    world, rank, local = dist_setup()
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    h = pmcmc.Handle(local)
    solve = lambda cs: pmcmc.fleet_solve(cs, workers=8, handle=h, errors="report")
    Dd.fleet_solve_distributed(chains, gather=False, solve=solve)  # warm-up
    times, mine = [], {}
    with ClockSampler(local) as clk:
        for _ in range(max(1, args.steps)):
            dist.barrier()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            mine = Dd.fleet_solve_distributed(chains, gather=False, solve=solve)
            torch.cuda.synchronize(dev)
            t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            times.append(float(t.item()))
    ok = torch.tensor([sum(chains[i][1].T for i, r in mine.items() if r[1]["converged"]),
                       sum(1 for r in mine.values() if r[1]["converged"]),
                       sum(1 for r in mine.values() if r[1]["status"] == 4)],
                      dtype=torch.float64, device=dev)
    dist.all_reduce(ok)
    best = min(times)
    clocks = clk.summary()
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return
    total_T = sum(s.T for _, s, *_ in chains)
    line = {"metric": METRIC, "secondary": True, "value": total_T / best, "unit": "samples/s",
            "n_gpus": world, "steps": len(times), "warmup": 1, "ms_per_step": 1e3 * best,
            "higher_is_better": True, "scaling": "strong", "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 per chain + counter-based Philox tape)",
            "timing": "host wall clock around each rank's share with device synchronisation, "
                      "max over ranks (all_reduce), best of the timed runs",
            "config": {"workload": workload, "chains": len(chains), "T_total": total_T,
                       "parallelism": f"chains partitioned over {world} GPUs (longest first)",
                       "converged": int(ok[1].item()), "nonfinite": int(ok[2].item()),
                       "T_converged": int(ok[0].item())},
            "clocks_rank0": clocks}
    print(json.dumps(line), flush=True)


def run_fleet_full(args):
    """All 512 chains of the uneven logistic fleet at full N and T (chain c: seed c,
    D uniform on {16, ..., 512}, N in [1000, 20000], T in [1024, 32768], :stoch_diag,
    eps adapted per chain from 0.5 / sqrt(D) by dual averaging over short blocks),
    solved through pmcmc_fleet_solve on 8 worker streams in batches of 64 chains
    (the data of all 512 would take ~11 GB of host memory); the plain per-chain
    FP32 path on 16 chains against the same chains on the fleet."""
    import numpy as np
    import torch

    import pmcmc
    from pmcmc import configs

    from pmcmc.adapt import adapt_fleet

    n_total, batch = (64, 32) if args.small else (512, 64)
    rounds, t_adapt = 12, 128
    h = pmcmc.Handle(0)
    pmcmc.fleet_solve(configs.logistic_fleet(n_chains=4, scale=0.05), workers=4, handle=h,
                      errors="report")  # warm-up
    per, total_s, adapt_s = [], 0.0, 0.0
    sub = None
    with ClockSampler(0) as clk:
        for b0 in range(0, n_total, batch):
            chains0 = configs.logistic_fleet(n_chains=min(batch, n_total - b0), first=b0)
            for m, *_ in chains0:  # device targets outside the timed region
                m.device_target(h)
            # per-chain step size: dual averaging from eps = 0.5 / sqrt(D) over short
            # blocks of the whole batch, the chain moving on from block to block
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            chains, hist = adapt_fleet(chains0, rounds=rounds, T_adapt=t_adapt, handle=h,
                                       method=args.adapt, target_accept=args.target_accept)
            torch.cuda.synchronize()
            adapt_s += time.perf_counter() - t0
            t0 = time.perf_counter()
            res = pmcmc.fleet_solve(chains, workers=8, handle=h, errors="report")
            torch.cuda.synchronize()
            total_s += time.perf_counter() - t0
            for (m, smp, *_), (_, s0, *_), r, hc in zip(chains, chains0, res, hist):
                per.append({"D": m.dim, "N": m.target["X"].shape[0], "T": smp.T,
                            "eps0": s0.epsilon, "eps": smp.epsilon,
                            "adapt_rates": [round(a, 3) for _, a in hc[-3:]],
                            "iters": r[1]["iters"], "converged": bool(r[1]["converged"]),
                            "status": r[1]["status"],
                            "accept": float(np.mean(r[3])) if r[3] is not None else None})
            if b0 == 0:
                sub = chains[:16]
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                rf = pmcmc.fleet_solve(sub, workers=8, handle=h, errors="report")
                torch.cuda.synchronize()
                sub_fleet = time.perf_counter() - t0
                plain = [(m, dataclasses.replace(smp, exec="plain"), *rest)
                         for m, smp, *rest in sub]
                t0 = time.perf_counter()
                rp = pmcmc.fleet_solve(plain, workers=1, handle=h, errors="report")
                torch.cuda.synchronize()
                sub_plain = time.perf_counter() - t0
                sub_T = sum(smp.T for _, smp, *_ in sub)
                sub_ok = [bool(a[1]["converged"]) and bool(b[1]["converged"])
                          for a, b in zip(rf, rp)]
                sub_stats = {"chains": len(sub), "T_total": sub_T,
                             "fleet": {"value": sub_T / sub_fleet, "unit": "samples/s",
                                       "converged": sum(bool(r[1]["converged"]) for r in rf)},
                             "plain_per_chain": {"value": sub_T / sub_plain, "unit": "samples/s",
                                                 "converged": sum(bool(r[1]["converged"])
                                                                  for r in rp)},
                             "speedup_fleet_over_plain": sub_plain / sub_fleet,
                             "both_converged": sum(sub_ok)}
                del rf, rp, plain
            del chains, res
    ok = [c for c in per if c["converged"] and c["status"] == 0]
    samples = sum(c["T"] for c in ok)
    line = {"metric": METRIC, "secondary": True, "value": samples / total_s, "unit": "samples/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * total_s,
            "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded NumPy PCG64 per chain + counter-based Philox tape)",
            "timing": "host wall clock around each batch's pmcmc_fleet_solve with device "
                      "synchronisation (host outputs), summed over the batches; only "
                      "converged chains count as samples; the step-size adaptation before "
                      "it is timed apart (adaptation_s, value_with_adaptation)",
            "adaptation_s": adapt_s,
            "value_with_adaptation": samples / (total_s + adapt_s),
            "config": {"workload": f"logistic_fleet_{n_total}chains_full", "chains": n_total,
                       "batch": batch, "workers": 8,
                       "adaptation": f"{args.adapt.replace('_', ' ')}, {rounds} rounds of "
                                     f"{t_adapt}-step blocks per chain from eps = 0.5 / sqrt(D)"
                                     + (f", target accept {args.target_accept}"
                                        if args.adapt == "dual_averaging" else ""),
                       "T_total_all": sum(c["T"] for c in per), "T_total_converged": samples,
                       "converged": len(ok),
                       "not_converged": sum(1 for c in per if not c["converged"] and
                                            c["status"] == 0),
                       "nonfinite": [i for i, c in enumerate(per) if c["status"] == 4],
                       "newton_iters": {"min": min(c["iters"] for c in per),
                                        "median": statistics.median(c["iters"] for c in per),
                                        "max": max(c["iters"] for c in per)},
                       "accept_rate_median": statistics.median(
                           c["accept"] for c in per if c["accept"] is not None),
                       "eps_over_eps0_median": statistics.median(c["eps"] / c["eps0"]
                                                                 for c in per)},
            "subset_vs_plain": sub_stats,
            "per_chain": per,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity leg (the FP64 sequential chain on the host)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary diagonal-Gaussian measurements")
    ap.add_argument("--workload", default="logistic_n10k_d256",
                    choices=["logistic_n10k_d256", "aniso_diag_d100", "corr_gauss_d64_full",
                             "logistic_fleet", "logistic_fleet_full", "logistic_adjoint"])
    ap.add_argument("--dim", type=int, default=256,
                    help="logistic workload: dimension D (256 < D <= 512 runs the wide "
                         "tensor-core pass); D != 256 or --small is a secondary line")
    ap.add_argument("--adapt", default="dual_averaging",
                    choices=["dual_averaging", "esjd_gradient"],
                    help="logistic_fleet_full: per-chain step-size adaptation before the solves")
    ap.add_argument("--target-accept", type=float, default=0.574,
                    help="logistic_fleet_full with dual averaging: the accept rate it targets")
    ap.add_argument("--small", action="store_true",
                    help="secondary workloads: shorter T for profiler captures")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "logistic_fleet":
        run_fleet(args)
    elif args.workload == "logistic_fleet_full":
        run_fleet_full(args)
    elif args.workload == "logistic_adjoint":
        run_adjoint(args)
    elif args.workload == "aniso_diag_d100":
        run_gauss(args)
    elif args.workload == "corr_gauss_d64_full" or args.small or args.dim != 256:
        run_secondary(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
