#!/usr/bin/env python
"""Benchmark: seconds per CCSD iteration on a seeded synthetic Hamiltonian.

One step = one CC iteration: the full CCSD formula (43 [ADD]/[CONTR] items,
every block contraction of every item on the device), energy and residual
norm read back, DIIS update of the amplitudes.  Default workload: closed-shell
CCSD, C1, n_occ=24, n_virt=200, n_aux=900 (the metric's headline size);
--config 0 selects n_occ=8, n_virt=32, n_aux=160.

The line's `value` is the iteration with FP64 emulated by four int8 slices
on the tensor cores (precision mode 3, the bulk mode of the mixed solve),
with `precision` giving its errors against FP64 from identical amplitudes,
`fp64` the plain FP64 iteration and `i8` / `tf32` the other tensor-core
modes measured in the same run; `use_tr` times the iteration with the
spin-flip symmetry the reference uses by default; `spin_prj` times the
singlet projection of the doubles residual against the HBM roofline;
`convergence` gives the time to |dE| < 1 uEh of FP64 and the mixed solves at
o24/v200 on a variant of the Hamiltonian whose CC iteration converges;
`d2h` times the CCSD iteration and `ccsdt` the CCSDT iteration (FP64, fixed
tile rule) on the CCSDT configuration's workload (D2h, o6/v48, naux 300).

--impl reference times the CPU restatement of the reference path (oracle/,
route 3: gather, ILP64 OpenBLAS dgemm on all host cores, scatter) on the same
workload and metric, each step a bounded sample of the block contractions
extrapolated to a full iteration (the line says so).

Multi-GPU (torchrun, one rank per GPU): one solve sharded over the ranks
(cc.Shard, owner-computes: every rank runs its share of the output tiles of
the residual and energy contractions, intermediates and amplitudes are
replicated, the residuals are summed by an NCCL all-reduce per iteration);
the value is the seconds per iteration of that solve, max over ranks
(strong scaling).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gecco-public_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# the contraction whose GEMM launch stands for the dominant kernel
ROOFLINE_CONTRACTION = "r2_ladder"

# DRAM traffic of the roofline launch per algorithmic byte (operands read
# once at 8 bytes per element, FP64 or split TF32 hi + lo, plus the result's
# read-modify-write), measured by ncu on the same launch at the reduced size
# o12/v100 (dram__bytes_read.sum + dram__bytes_write.sum of k_gemm_tc and of
# k_gemm<128,64>: 1.2436 GB and 1.2470 GB against 1.2423 GB of algorithmic
# bytes); the full-size traffic is this ratio times the full-size
# algorithmic bytes
TRAFFIC_PER_ALGORITHMIC_BYTE = {"k_gemm_tc": 1.2436 / 1.2423, "k_gemm": 1.2470 / 1.2423,
                                # four int8 slices (4 bytes per operand element):
                                # k_gemm_i8<4,128> at o12/v100, 0.6385 GB
                                # against 0.6379 GB
                                "k_gemm_i8_4": 0.6385 / 0.6379}

SIGMA_SPEC = 0.05
CONFIGS = {
    0: dict(nocc=8, nvir=32, naux=160, seed=1000, sigma=SIGMA_SPEC,
            name="CCSD C1 o8 v32 naux160", tag="ccsd_o8v32"),
    # the sizes and point group of the CCSDT configuration (D2h, irreps
    # round-robin), run with the CCSD formula: thousands of uneven
    # symmetry / spin blocks per iteration
    1: dict(nocc=6, nvir=48, naux=300, seed=1001, sigma=SIGMA_SPEC, nsym=8,
            name="CCSD D2h o6 v48 naux300", tag="ccsd_d2h_o6v48"),
    2: dict(nocc=24, nvir=200, naux=900, seed=1002, sigma=SIGMA_SPEC,
            name="CCSD C1 o24 v200 naux900", tag="ccsd_o24v200"),
    # reduced size of the same family, used for kernel captures (a few GB)
    10: dict(nocc=12, nvir=100, naux=450, seed=1010, sigma=SIGMA_SPEC,
             name="CCSD C1 o12 v100 naux450", tag="ccsd_o12v100"),
    # the o24/v200 shape with a smaller standard deviation of B: with
    # sigma = 0.05 at naux = 900 the exchange integrals naux*sigma^2 are
    # 2.25 Eh, above most orbital gaps, and the CC iteration diverges, as it
    # does at 0.0211 (the o8/v32 value of naux*sigma^2) and at 0.013; at
    # 0.007 plain FP64 diagonal + DIIS converges to a residual norm of 1e-9
    # in about 40 iterations
    12: dict(nocc=24, nvir=200, naux=900, seed=1002, sigma=0.007,
             name="CCSD C1 o24 v200 naux900, B std 0.007", tag="ccsd_o24v200_conv"),
}


def metric_of(cfg):
    """the metric string of both arms (same workload, same unit)"""
    return f"s/CC-iteration ({cfg['name']})"


def clocks_sampler(stop, out, index):
    cmd = ["nvidia-smi", f"--id={index}",
           "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits"]
    while not stop.is_set():
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=5).stdout.strip()
            if r:
                out.append([x.strip() for x in r.split(",")])
        except Exception:
            pass
        stop.wait(0.2)


def clock_summary(samples):
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"]}
    sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
    mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
    reasons = set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for s in samples:
        for k, n in enumerate(names):
            if len(s) > 4 + k and s[4 + k].lower() == "active":
                reasons.add(n)
    return {"sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons)}


def fp64_peak():
    """measured FP64 tensor peak: cuBLAS DGEMM 8192^3, best of 5"""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def setup_hamiltonian(cfg):
    import hamiltonian as hm
    return hm.synthetic(cfg["nocc"], cfg["nvir"], cfg["naux"], seed=cfg["seed"],
                        sigma=cfg["sigma"], nsym=cfg.get("nsym", 1))


def data_desc(cfg):
    return (f"synthetic (seeded Hamiltonian: eps_occ~U[-1.5,-0.3], eps_virt~U[0.1,4.0], "
            f"B_pq (p<=q, mirrored)~N(0,{cfg['sigma']:.4g}^2))")


def cpu_baseline_oracle(sp, eps, B, target_s, cores, host_lists):
    """the oracle (route 3, OpenBLAS on all host cores) on the same workload:
    every formula item, only every stride-th long-operand batch executed;
    returns seconds per full iteration (extrapolated) and the sample
    description"""
    import binding
    import cc
    from engine import OracleEngine
    import hamiltonian as hm
    binding.set_blas(cores)
    oe = OracleEngine(route=3)
    s = cc.CCSolver(oe, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
    for name, x in host_lists.items():
        oe.data[s.lid(name)][:] = x
    # calibrate the stride on a short probe, then time one sampled iteration
    stride = 4096
    binding.sampling(stride)
    t0 = time.time()
    s.evaluate()
    est_full = binding.scaled_time(time.time() - t0, binding.sampling_report())
    stride = int(max(1, min(stride, est_full / max(target_s, 1e-3))))
    binding.sampling(stride)
    t0 = time.time()
    s.evaluate()
    wall = time.time() - t0
    rep = binding.sampling_report()
    scaled = binding.scaled_time(wall, rep)
    binding.sampling(1)
    sample = (f"one CCSD iteration of the same workload through the oracle (route 3 gathers, "
              f"OpenBLAS dgemm, scatters) with every {stride}-th of {rep['batches']} "
              f"long-operand batches executed ({rep['done']} run, {wall:.1f} s wall), "
              f"extrapolated by batch count")
    return scaled, sample


def evaluation_errors(eng, solver, mode=1):
    """one formula evaluation in precision `mode` and one in FP64 from the
    same amplitudes (the solver's current T1, T2): errors of the mode's
    energy, residuals and next Jacobi step against FP64"""
    import torch
    from devfill import list_tensor

    def lists(names):
        return {n: list_tensor(eng, solver.lid(n), solver.lists[n][1]).clone()
                for n in names}

    out = {}
    for m in (mode, 0):
        eng.set_precision(m)
        solver.evaluate()
        eng.sync()
        out[m] = lists(["E", "R1", "R2"])
    eng.set_precision(mode)
    d = {n: list_tensor(eng, solver.lid(n), solver.lists[n][1]) for n in ("DT1", "DT2")}
    res = {"dE": abs(float(out[mode]["E"][0] - out[0]["E"][0])), "E_fp64": float(out[0]["E"][0])}
    num, den = 0.0, 0.0
    for a, r in (("T1", "R1"), ("T2", "R2")):
        x1, x0 = out[mode][r], out[0][r]
        res[f"d{r}_max_rel"] = float((x1 - x0).abs().max() / x0.abs().max().clamp_min(1e-300))
        res[f"d{r}_norm_rel"] = float((x1 - x0).norm() / x0.norm().clamp_min(1e-300))
        # the next diagonal step -R/D: the amplitude change the error reaches
        dd = d["D" + a].abs().clamp_min(1e-10) * torch.sign(d["D" + a])
        s1, s0 = -x1 / dd, -x0 / dd
        num += float((s1 - s0).norm() ** 2)
        den += float(s0.norm() ** 2)
    res["step_norm_rel"] = math.sqrt(num / max(den, 1e-300))
    return res


def run_gpu(args, cfg):
    import torch

    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.only_convergence:
        cfgc = dict(CONFIGS[args.conv_config])
        if args.conv_sigma:
            cfgc["sigma"] = args.conv_sigma
            cfgc["name"] += f" (B std {args.conv_sigma})"
        variants = json.loads(args.conv_variants) if args.conv_variants else None
        print(json.dumps({"convergence": convergence(local, cfgc, maxiter=args.conv_maxiter,
                                                     variants=variants)}), flush=True)
        return
    tracing = args.trace_contraction or args.trace_learned or args.trace_spin_prj
    peak = fp64_peak() if rank == 0 and not tracing else None
    sp, eps, B = setup_hamiltonian(cfg)
    eng = gccu.Engine(local)
    eng.set_precision(args.precision)
    eng.set_tuning(args.tune)
    solver = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                         shard=cc.Shard(dist) if dist else None)
    t0 = time.time()
    solver.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
    setup_s = time.time() - t0
    if args.trace_learned:
        # the learned step once on the doubles lists (the command profilers
        # capture): random residual and previous step, the denominators
        import learned
        for name, seed in (("R2", 1), ("PT2", 2)):
            lid, n, _ = solver.lists[name]
            x = np.random.default_rng(seed).standard_normal(n) * 1e-3
            eng.upload(lid, x)
        eng.lp_set_weights(learned.initial_weights(3))
        eng.event_record(0)
        eng.lp_precondition(solver.lid("ST2"), solver.lid("R2"), solver.lid("DT2"),
                            solver.lid("PT2"), fac=-1.0)
        eng.event_record(1)
        ms = eng.event_elapsed(0, 1)
        n = solver.lists["T2"][1]
        eng.close()
        print(json.dumps({"trace": "learned step", "workload": cfg["name"], "elements": n,
                          "ms": ms, "GB_per_s": 32.0 * n / (ms * 1e-3) / 1e9}), flush=True)
        return
    if args.trace_spin_prj:
        # the singlet projection of the doubles residual (the command the
        # profilers capture)
        singlet_residuals(eng, solver)
        out = measure_spin_prj(eng, solver, reps=3)
        eng.close()
        print(json.dumps({"trace": "spin projection", "workload": cfg["name"], **out}),
              flush=True)
        return
    if args.trace_contraction:
        # one formula item, run once eagerly (the command profilers capture)
        items = [it for it in solver.formula if it.get("name") == args.trace_contraction]
        if not items:
            raise SystemExit(f"no formula item named {args.trace_contraction!r}")
        eng.event_record(0)
        solver.run_item(items[0])
        eng.event_record(1)
        ms = eng.event_elapsed(0, 1)
        eng.close()
        print(json.dumps({"trace": args.trace_contraction, "workload": cfg["name"],
                          "ms_including_planning": ms}), flush=True)
        return
    modes = [args.precision] + ([0] if args.precision != 0 and not args.no_fp64 else [])
    results = {}
    for mode in modes:
        reset_amplitudes(eng, solver)
        eng.set_precision(mode)
        results[mode] = measure(args, cfg, eng, solver, local, dist, mode, main=True)
    r = results[modes[0]]
    line = {
        "metric": metric_of(cfg),
        "value": r["ms"] / 1e3,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms"],
        "higher_is_better": False,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None,
        "dtype": DTYPE[modes[0]],
        "data": data_desc(cfg) + "; inputs larger than L2 (two-electron list "
                f"{8 * solver.lists['V'][1] / 1e9:.1f} GB)",
        "config": {"workload": cfg["name"], "method": "CCSD spin-orbital, DIIS maxsub 8",
                   "nocc": cfg["nocc"], "nvirt": cfg["nvir"], "naux": cfg["naux"],
                   "sigma_B": cfg["sigma"], "use_tr": False,
                   "parallelism": (f"owner-computes sharding x{world}, NCCL all-reduce of "
                                   "the residuals" if world > 1 else "single GPU"),
                   "l2": "inputs > L2", "setup_s": round(setup_s, 2),
                   "energy_last": r["energies"][-1]},
        "roofline": roofline(r, peak, modes[0], solver, eng),
        "clocks": clock_summary(r["samples"]),
        "e2e": r["e2e"],
        "gpu_launches": r["launches"],
    }
    if 0 in results and modes[0] != 0:
        f = results[0]
        line["fp64"] = {"metric": metric_of(cfg) + " plain FP64", "value": f["ms"] / 1e3,
                        "ms_per_step": f["ms"], "e2e": f["e2e"], "gpu_launches": f["launches"],
                        "roofline": roofline(f, peak, 0, solver, eng),
                        "clocks": clock_summary(f["samples"]),
                        "energy_last": f["energies"][-1]}
    if 0 in results and modes[0] != 0 and world == 1:
        # errors of one evaluation in the tensor-core modes against FP64 from
        # identical amplitudes: those after two plain Jacobi iterations from zero
        reset_amplitudes(eng, solver)
        eng.set_precision(0)
        for _ in range(2):
            solver.iterate()
            solver.step()
        line["precision"] = dict(
            evaluation_errors(eng, solver, modes[0]),
            amplitudes="after two FP64 Jacobi iterations from T=0",
            note=f"evaluation with {METRIC_MODE[modes[0]]} minus FP64 evaluation; "
                 "R*_max_rel relative to max|R|")

    # side measurements: on one GPU a failure in one of them is recorded in
    # its own field and the headline line is still printed; sharded runs keep
    # every rank on the same collective steps and let an error end the run
    def side(key, fn, sub=None):
        target = line if sub is None else line[sub]
        if world > 1:
            target[key] = fn()
            return
        try:
            target[key] = fn()
        except Exception as ex:  # noqa: BLE001 - reported in the bench line
            target[key] = {"error": f"{type(ex).__name__}: {ex}"[:400]}

    if world == 1 and not args.no_spin_prj:
        side("spin_prj", lambda: (singlet_residuals(eng, solver),
                                  measure_spin_prj(eng, solver))[1])

    if args.tune:
        rows = eng.tuning_report()
        line["tuning"] = {
            "mode": "autotuned at each contraction's first call (warm-up), cached per "
                    "block-shape histogram",
            "histograms": len(rows),
            "non_default_choices": int(sum(r[1] != 0 for r in rows)),
            "rows": [{"block_contractions": int(r[0]), "chosen": int(r[1]),
                      "ms": [round(x, 4) for x in r[2:] if x >= 0]} for r in rows]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        host_lists = {}
        for name in ("F", "V", "T1", "T2", "DT1", "DT2"):
            lid, n, _ = solver.lists[name]
            x = np.empty(n)
            eng.get_vec(lid, 0, x.ctypes.data, n)
            host_lists[name] = x
        cores = os.cpu_count()
        val, sample = cpu_baseline_oracle(sp, eps, B, args.cpu_seconds, cores, host_lists)
        line["cpu_baseline"] = {"value": val, "unit": "s", "cores": cores, "kind": "port",
                                "sample": sample}
    eng.close()
    del solver
    torch.cuda.empty_cache()
    if args.precision != 0 and not args.no_i8:
        # the other tensor-core modes, each on an engine of its own
        for mode in (3, 2, 1):
            if mode != args.precision:
                side(MODE_LABEL[mode],
                     lambda mode=mode: measure_i8(args, cfg, local, dist, peak, mode))
    if args.tune and world == 1 and not args.no_fixed_rule:
        side("fixed_rule", lambda: measure_fixed_rule(args, cfg, local, modes[0]), "tuning")
    if not args.no_d2h and world == 1:
        side("d2h", lambda: measure_d2h(args, local))
    if not args.no_use_tr and world == 1:
        side("use_tr", lambda: measure_use_tr(args, cfg, local, dist, modes,
                                              {m: results[m]["energies"] for m in modes}))
    weights = None
    if rank == 0 and world == 1 and not args.no_learned:
        side("learned", lambda: learned_stream(local, args.c4_train, args.c4_test))
        if isinstance(line["learned"], tuple):
            line["learned"], weights = line["learned"]
    if rank == 0 and world == 1 and not args.no_convergence:
        side("convergence", lambda: convergence(local, CONFIGS[args.conv_config], weights,
                                                maxiter=args.conv_maxiter))
        side("convergence_small", lambda: convergence(local, CONFIGS[0], weights))
    if not args.no_ccsdt and world == 1:
        side("ccsdt", lambda: measure_ccsdt(args, local))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


METRIC_MODE = {0: "plain FP64", 1: "split TF32 on the tensor cores (FP32 accumulation per "
                                   "4096-index chunk, FP64 sums)",
               2: "FP64 emulated with five int8 slices on the tensor cores",
               3: "FP64 emulated with four int8 slices on the tensor cores"}
MODE_LABEL = {0: "fp64", 1: "tf32", 2: "i8", 3: "i8_fast"}
DTYPE = {0: "f64", 1: "tf32x3 products, f32 accumulate per 4096-chunk, f64 sums",
         2: "s8 slices x5 (15 products), s32 exact accumulate, f64 combine",
         3: "s8 slices x4 (10 products), s32 exact accumulate, f64 combine"}
SLICE_PRODUCTS = {2: 15, 3: 10}


def measure_spin_prj(eng, solver, reps=10):
    """singlet projection (gccu_spin_prj_list, one k_spin_prj launch) of the
    doubles residual list of the benchmark: ms per projection (median of
    reps, L2 flushed before each), achieved HBM bandwidth for its algorithmic
    bytes (16 per element: one read, one write), and two size-independent
    checks -- the closed-shell residual is a singlet (the projection leaves it
    unchanged) and the projection of a random list is idempotent"""
    import torch
    lid, n, _ = solver.lists["R2"]
    r0 = eng.download(lid, n)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    eng.spin_prj(lid)  # plans the list
    moved = float(np.abs(eng.download(lid, n) - r0).max() / max(np.abs(r0).max(), 1e-300))
    times = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        eng.sync()
        eng.event_record(0)
        eng.spin_prj(lid)
        eng.event_record(1)
        times.append(eng.event_elapsed(0, 1))
    x = np.random.default_rng(12).standard_normal(n)
    eng.upload(lid, x)
    eng.spin_prj(lid)
    y = eng.download(lid, n)
    eng.spin_prj(lid)
    z = eng.download(lid, n)
    eng.upload(lid, r0)
    del flush
    ms = float(np.median(times))
    peak, src = measured_bf16_tflops("hbm_gbs")
    gbs = 16.0 * n / (ms * 1e-3) / 1e9
    return {"list": "R2 (PP;HH), FP64", "elements": n, "ms": ms,
            "algorithmic_bytes": 16 * n, "achieved_GBps": gbs, "peak_GBps": peak,
            "peak_source": src + " HBM copy", "frac": gbs / peak,
            "singlet_residual_change_rel": moved,
            "random_list_change_rel": float(np.abs(y - x).max() / np.abs(x).max()),
            "idempotence_rel": float(np.abs(z - y).max() / np.abs(y).max())}


def singlet_residuals(eng, solver):
    """residuals of singlet amplitudes: two FP64 Jacobi steps from T = 0 and
    one more evaluation"""
    reset_amplitudes(eng, solver)
    eng.set_precision(0)
    for _ in range(2):
        solver.iterate()
        solver.step()
    solver.iterate()


def reset_amplitudes(eng, solver):
    """zero amplitudes, a fresh DIIS subspace and no captured graph"""
    for a in solver.amps:
        eng.zero(solver.lid(a))
    if hasattr(solver, "_diis"):
        del solver._diis
    solver.graph = None


def max_over_ranks(value, dist):
    """the largest of every rank's value (the job's time is its slowest
    rank's); NCCL reduces a device tensor, gloo a host one; without a process
    group the value itself"""
    if dist is None:
        return value
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measure(args, cfg, eng, solver, local, dist, mode, steps=None, profile=True, e2e=True,
            main=False):
    """warm-up (plans every contraction in this precision mode), the timed
    graph-replayed iterations, one eagerly profiled iteration and the
    end-to-end iterations through host buffers"""
    import torch

    steps = steps or args.steps
    energies = []
    for _ in range(args.warmup):
        en, rn = solver.iterate()
        energies.append(en)
        solver.diis_step()
    solver.capture()
    eng.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stop, samples = threading.Event(), []
    th = threading.Thread(target=clocks_sampler, args=(stop, samples, local), daemon=True)
    th.start()
    eng.reset_stats()
    if main:  # the range a profiler's launch list can be limited to (--nvtx-include timed/)
        torch.cuda.nvtx.range_push("timed")
    eng.event_record(0)
    for _ in range(steps):
        en, rn = solver.iterate()
        energies.append(en)
        solver.diis_step()
    eng.event_record(1)
    if main:
        torch.cuda.nvtx.range_pop()
    ms_total = eng.event_elapsed(0, 1)
    stop.set()
    th.join()
    _, launches = eng.stats()
    ms = max_over_ranks(ms_total / steps, dist)
    out = {"ms": ms, "launches": int(launches), "samples": samples, "energies": energies}
    if profile:
        # per-kernel times: one more iteration, launched eagerly with every
        # [CONTR] kernel bracketed by events on the engine's stream (outside
        # the timed loop)
        eng.profile(True)
        solver.evaluate()
        prof = eng.profile_report()
        eng.profile(False)
        names = [it["name"] for it in solver.formula if it["kind"] == "CONTR"]
        if len(names) != len(prof):
            raise RuntimeError(f"profile rows ({len(prof)}) do not match contractions "
                               f"({len(names)})")
        if (args.profile_out and main and mode == args.precision and
                int(os.environ.get("RANK", 0)) == 0):
            with open(args.profile_out, "w") as f:
                json.dump([{"item": n, "gflop": r[0] / 1e9, "ms": r[2] / max(r[1], 1),
                            "tflops": (r[0] / (r[2] / max(r[1], 1) * 1e-3) / 1e12
                                       if r[2] else None),
                            "block_contractions": int(r[3]), "tiles": int(r[4]),
                            "pack_ms": r[5] / max(r[1], 1)}
                           for n, r in zip(names, prof)], f, indent=1)
        out.update(prof=prof, names=names)
    if e2e:
        out["e2e"] = measure_e2e(args, eng, solver)
    return out


def measure_e2e(args, eng, solver):
    """the same iteration through the public API with host buffers: the
    amplitudes come from pinned host memory, the residuals and the energy go
    back"""
    import torch

    nT = {a: solver.lists[a][1] for a in solver.amps}
    nR = {a: solver.lists[solver.res[a]][1] for a in solver.amps}
    host_t = {a: torch.empty(n, dtype=torch.float64, pin_memory=True) for a, n in nT.items()}
    host_r = {a: torch.empty(n, dtype=torch.float64, pin_memory=True) for a, n in nR.items()}
    for a in solver.amps:
        eng.get_vec(solver.lid(a), 0, host_t[a].data_ptr(), nT[a])
    e2e_steps = max(1, min(args.steps, 5))
    eng.sync()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for a in solver.amps:
            eng.put_vec(solver.lid(a), 0, host_t[a].data_ptr(), nT[a])
        solver.iterate()
        for a in solver.amps:
            eng.get_vec(solver.lid(solver.res[a]), 0, host_r[a].data_ptr(), nR[a])
    eng.sync()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    return {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * sum(nT.values()),
            "d2h_bytes_per_step": 8 * sum(nR.values()) + 8}


def measure_i8(args, cfg, local, dist, peak, mode):
    """seconds per iteration in a tensor-core precision mode (1: split TF32,
    2: five int8 slices, 3: four) on an engine of its own (the plans and
    cached operand panels of several precision modes do not fit one device
    together), its roofline launch, and the errors of one evaluation against
    FP64 from identical amplitudes"""
    import torch

    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    sp, eps, B = setup_hamiltonian(cfg)
    eng = gccu.Engine(local)
    try:
        eng.set_tuning(args.tune)
        s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                        shard=cc.Shard(dist) if dist else None)
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        eng.set_precision(mode)
        f = measure(args, cfg, eng, s, local, dist, mode, main=True)
        out = {"metric": metric_of(cfg) + f" {METRIC_MODE[mode]}",
               "value": f["ms"] / 1e3, "unit": "s", "ms_per_step": f["ms"], "e2e": f["e2e"],
               "gpu_launches": f["launches"], "dtype": DTYPE[mode],
               "roofline": roofline(f, peak, mode, s, eng),
               "clocks": clock_summary(f["samples"]),
               "energy_last": f["energies"][-1]}
        if dist is None:
            reset_amplitudes(eng, s)
            eng.set_precision(0)
            for _ in range(2):
                s.iterate()
                s.step()
            out["precision"] = dict(
                evaluation_errors(eng, s, mode),
                amplitudes="after two FP64 Jacobi iterations from T=0",
                note=f"evaluation with {METRIC_MODE[mode]} minus FP64 evaluation; "
                     "R*_max_rel relative to max|R|")
    finally:
        eng.close()
        torch.cuda.empty_cache()
    return out


def measure_use_tr(args, cfg, local, dist, modes, plain_energies):
    """seconds per iteration with spin-flip symmetry (calculate.routes.use_tr,
    the reference's default): half of the Ms cases of every contraction into
    a spin-symmetric list, doubled, then symmetrised (sym_ab_blk); the first
    warm-up energies are compared with those of the plain evaluation (same
    iterates from T = 0)"""
    import torch

    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    sp, eps, B = setup_hamiltonian(cfg)
    eng = gccu.Engine(local)
    out = {}
    try:
        s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd", use_tr=True)
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        for mode in modes:
            reset_amplitudes(eng, s)
            eng.set_precision(mode)
            r = measure(args, cfg, eng, s, local, dist, mode, steps=max(2, args.steps // 2),
                        profile=False, e2e=False)
            ref = plain_energies[mode]
            k = min(3, len(ref), len(r["energies"]))
            out[MODE_LABEL[mode]] = {
                "value": r["ms"] / 1e3, "unit": "s", "gpu_launches": r["launches"],
                "clocks": clock_summary(r["samples"]),
                "dE_first_iterations_vs_plain": max(
                    abs(a - b) for a, b in zip(r["energies"][:k], ref[:k]))}
    finally:
        eng.close()
        torch.cuda.empty_cache()
    return out


def measure_fixed_rule(args, cfg, local, mode):
    """seconds per iteration of the headline mode with the fixed tile rule
    (no autotuning), in a fresh engine on the same Hamiltonian"""
    import torch

    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    sp, eps, B = setup_hamiltonian(cfg)
    eng = gccu.Engine(local)
    try:
        eng.set_precision(mode)
        eng.set_tuning(0)
        s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        r = measure(args, cfg, eng, s, local, None, mode, steps=max(2, args.steps // 2),
                    profile=False, e2e=False)
        return {"value": r["ms"] / 1e3, "unit": "s", "clocks": clock_summary(r["samples"])}
    finally:
        eng.close()
        torch.cuda.empty_cache()


def measure_ccsdt(args, local):
    """the CCSDT iteration (cc.excitation_formula: the connected terms as 102
    chains of binary contractions, 143 [CONTR] per evaluation) on the CCSDT
    configuration's workload (D2h, o6/v48, naux 300) in FP64 with the fixed
    tile rule: seconds per iteration, block contractions, flops and kernel
    launches per iteration"""
    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    cfg = CONFIGS[1]
    sp, eps, B = setup_hamiltonian(cfg)
    eng = gccu.Engine(local)
    try:
        eng.set_precision(0)
        eng.set_tuning(0)
        t0 = time.perf_counter()
        s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsdt")
        s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
        steps = min(args.steps, 5)
        r = measure(args, cfg, eng, s, local, None, 0, steps=steps, profile=True, e2e=False)
        prof = r["prof"]
        en = r["energies"][-1]
        return {"workload": cfg["name"].replace("CCSD", "CCSDT", 1),
                "method": "CCSDT, unfactorised connected terms",
                "precision": "FP64", "tile_rule": "fixed", "value": r["ms"] / 1e3, "unit": "s",
                "steps": steps, "contractions": len(r["names"]),
                "block_contractions": int(np.sum(prof[:, 3])),
                "gflop_per_iteration": float(np.sum(prof[:, 0])) / 1e9,
                "launches_per_iteration": r["launches"] / max(steps, 1),
                "energy_last": en if math.isfinite(en) else None,
                "wall_s_with_planning": round(time.perf_counter() - t0, 2),
                "clocks": clock_summary(r["samples"])}
    finally:
        eng.close()


def measure_d2h(args, local):
    """the CCSD iteration on the D2h workload (the CCSDT configuration's sizes
    and point group) in split TF32, with the fixed tile rule and autotuned:
    seconds per iteration, block contractions and kernel launches per
    iteration"""
    import torch

    import cc
    import gccu
    from devfill import TorchIntegrals
    import hamiltonian as hm

    cfg = CONFIGS[1]
    sp, eps, B = setup_hamiltonian(cfg)
    out = {"workload": cfg["name"], "precision": "split TF32"}
    for tune in (0, 1):
        eng = gccu.Engine(local)
        try:
            eng.set_precision(1)
            eng.set_tuning(tune)
            s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            r = measure(args, cfg, eng, s, local, None, 1, steps=args.steps, profile=True,
                        e2e=False)
            items = int(np.sum(r["prof"][:, 3]))
            out["autotuned" if tune else "fixed_rule"] = {
                "value": r["ms"] / 1e3, "unit": "s", "block_contractions": items,
                "launches_per_iteration": r["launches"] / max(args.steps, 1),
                "energy_last": r["energies"][-1]}
            if tune:
                out["histograms_tuned"] = len(eng.tuning_report())
        finally:
            eng.close()
            torch.cuda.empty_cache()
    return out


def plan_rows(eng, solver, name):
    it = [x for x in solver.formula if x.get("name") == name][0]
    o1, o2, r = solver.blk(it["op1"]), solver.blk(it["op2"]), solver.blk(it["res"])
    c = np.asarray(it["cnt"])
    ex1 = np.asarray(it["op1"][1]) - c
    ex2 = np.asarray(it["op2"][1]) - np.concatenate([c[4:], c[:4]])
    return eng.plan_items(o1, o2, r, ex1, ex2, c)


def roofline(r, fp64_peak_tflops, mode, solver, eng):
    """dominant kernel: the GEMM launch(es) of the pp-ladder contraction (the
    leading term; no operand gathers), timed with events in the profiled
    iteration: k_gemm<128,64> (FP64 DMMA) in mode 0, k_gemm_tc (split TF32 on
    tcgen05) in mode 1, k_gemm_i8 (int8 slices on tcgen05) in modes 2 and 3"""
    names, prof = r["names"], r["prof"]
    dom = prof[names.index(ROOFLINE_CONTRACTION)]
    dom_ms = (dom[2] - dom[5]) / dom[1]
    achieved = dom[0] / (dom_ms * 1e-3) / 1e12
    total_flops = float(np.sum(prof[:, 0] * prof[:, 1]))
    rows = plan_rows(eng, solver, ROOFLINE_CONTRACTION).astype(float)
    M, N, K = rows[:, 0], rows[:, 1], rows[:, 2]
    # operands read once (8 bytes per element in FP64 and split TF32, one byte
    # per slice with int8 slices), the result read and written
    op_bytes = {2: 5, 3: 4}.get(mode, 8)
    alg_bytes = float(op_bytes * np.sum(M * K + N * K) + 16 * np.sum(M * N))
    out = {"bound": "tensor", "achieved": achieved, "unit": "TFLOP/s",
           "flops_per_launch": dom[0], "ms_per_launch": dom_ms,
           "iteration_flops": total_flops,
           "iteration_tflops": total_flops / (r["ms"] * 1e-3) / 1e12,
           "algorithmic_bytes_per_launch": alg_bytes}
    kern = {0: "k_gemm", 1: "k_gemm_tc", 2: "k_gemm_i8_5", 3: "k_gemm_i8_4"}[mode]
    if kern in TRAFFIC_PER_ALGORITHMIC_BYTE:
        out["traffic"] = TRAFFIC_PER_ALGORITHMIC_BYTE[kern] * alg_bytes
        out["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
                                 "same launch at o12/v100 per algorithmic byte, times this "
                                 "launch's algorithmic bytes")
    else:
        out["traffic"] = None
    if mode in SLICE_PRODUCTS:
        # int8 dense peak = 2 x dense BF16 on B200; 15 (10) slice products per
        # useful FP64 product with five (four) slices
        npr = SLICE_PRODUCTS[mode]
        burst, src = measured_bf16_tflops("bf16_tflops")
        sustained, _ = measured_bf16_tflops("bf16_tflops_sustained")
        out.update(peak=burst * 2.0 / npr,
                   kernel=f"k_gemm_i8 {npr} int8 slice products (tcgen05 kind::i8, "
                          f"persistent), launch of [CONTR] {ROOFLINE_CONTRACTION}",
                   peak_source=f"of {src}: bf16_tflops x 2 (dense int8 = twice dense BF16) "
                               f"/ {npr} (slice products per useful product)",
                   frac_of_sustained=achieved / (sustained * 2.0 / npr))
        out["ladder_with_split_tflops"] = dom[0] / (dom[2] / dom[1] * 1e-3) / 1e12
    elif mode == 0:
        out.update(peak=fp64_peak_tflops,
                   kernel=f"k_gemm<128,64> FP64 DMMA, launch of [CONTR] {ROOFLINE_CONTRACTION}",
                   peak_source="cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in "
                               "MEASURED_PEAKS.json)")
    else:
        # the launch is timed on its own (events around it in an eager
        # iteration), so the burst BF16 figure is the denominator; the
        # fraction of the sustained (power-capped) figure is given beside it
        burst, src = measured_bf16_tflops("bf16_tflops")
        sustained, _ = measured_bf16_tflops("bf16_tflops_sustained")
        out.update(peak=burst / 6.0,
                   kernel=f"k_gemm_tc split TF32 (tcgen05, persistent), launch of [CONTR] "
                          f"{ROOFLINE_CONTRACTION}",
                   peak_source=f"of {src}: bf16_tflops / 2 (dense TF32 = half of dense BF16) "
                               "/ 3 (three TF32 products per useful product)",
                   frac_of_sustained=achieved / (sustained / 6.0))
        # the ladder end to end, its operand split included
        out["ladder_with_split_tflops"] = dom[0] / (dom[2] / dom[1] * 1e-3) / 1e12
    out["frac"] = (achieved / out["peak"]) if out["peak"] else None
    return out


# earlier measurement on this pool's B200s, used only when MEASURED_PEAKS.json
# (written before each run) is absent
FALLBACK_PEAKS = {"bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "hbm_gbs": 6650.0}


def measured_bf16_tflops(key="bf16_tflops"):
    """(value, "measured" from MEASURED_PEAKS.json | "fallback")"""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))[key]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_PEAKS[key], "fallback"


def convergence(local, cfg, weights=None, maxiter=80, variants=None):
    """time to |dE| < 1 uEh against the converged FP64 energy, per solve
    variant: plain FP64 ("fp64"), four int8 slices until the residual norm
    is below 1e-7 and five after it ("mixed"), four slices throughout
    ("i8_fast"), five throughout ("i8"), split TF32 until 1e-4 and five
    slices after it ("mixed_tf32") and, given weights, "mixed" with the
    learned step ("mixed_learned"); `variants` adds labels: options of
    CCSolver.solve_mixed, or {"plain": mode} for one precision throughout.
    Each variant is solved twice on one engine: from its first call, with
    every contraction planned and autotuned during the first iteration of
    each precision mode ("s_to_1uEh"), then again from zero amplitudes with
    the plans made ("s_to_1uEh_planned").  Wall time of the solve loop
    (device work, energy and residual reads, DIIS solves), graphs replayed
    after the first iteration of each mode; Hamiltonian set-up excluded."""
    import cc
    import gccu
    import hamiltonian as hm
    from devfill import TorchIntegrals

    mixed = {"schedule": [(3, 1e-7), (2, None)]}
    runs = {"fp64": {"plain": 0}, "mixed": dict(mixed), "i8_fast": {"plain": 3},
            "i8": {"plain": 2}, "mixed_tf32": {"schedule": [(1, 1e-4), (2, None)]}}
    if weights is not None:
        runs["mixed_learned"] = dict(mixed, learned=True)
    runs.update(variants or {})
    sp, eps, B = setup_hamiltonian(cfg)
    out = {"workload": cfg["name"], "sigma_B": cfg["sigma"],
           "variants": {k: {o: v for o, v in opts.items()} for k, opts in runs.items()}}
    ref = None
    ref_t = None

    def solve(s, eng, opts):
        hist = []
        t0 = time.perf_counter()

        def cb(it, en, rn):
            hist.append((it, en, rn, time.perf_counter() - t0))

        if "plain" in opts:
            eng.set_precision(opts["plain"])
            s.solve(maxiter=maxiter, conv=1e-9, use_graph=True, callback=cb)
        else:
            s.solve_mixed(maxiter=maxiter, conv=1e-9, callback=cb,
                          **{o: v for o, v in opts.items() if o != "learned"})
        eng.set_precision(0)
        return hist

    def hit(hist):
        return next((h for h in hist if abs(h[1] - ref) < 1e-6), None) if ref is not None else None

    for label, opts in runs.items():
        eng = gccu.Engine(local)
        try:
            s = cc.CCSolver(eng, hm.FactorizedIntegrals(sp, eps, B), method="ccsd",
                            learned=weights if opts.get("learned") else None)
            s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
            eng.sync()
            hist = solve(s, eng, opts)
            t = {a: eng.download(s.lid(a), s.lists[a][1]) for a in s.amps}
            switched = getattr(s, "switched_at", None)
            fallbacks = getattr(s, "fallbacks", None)
            planning = eng.plan_stats()
            if ref is None:
                ref = hist[-1][1]
                ref_t = t
            reset_amplitudes(eng, s)
            s.history = []
            hist_p = solve(s, eng, opts)
        finally:
            eng.close()
        h, hp = hit(hist), hit(hist_p)
        r = {"iterations": hist[-1][0], "energy": hist[-1][1], "residual": hist[-1][2],
             "s_total": hist[-1][3], "converged": hist[-1][2] < 1e-9,
             "iterations_to_1uEh": h[0] if h else None, "s_to_1uEh": h[3] if h else None,
             "s_first_iteration": hist[0][3],
             "s_to_1uEh_planned": hp[3] if hp else None,
             "s_total_planned": hist_p[-1][3], "iterations_planned": hist_p[-1][0],
             "s_per_iteration_planned": (hist_p[-1][3] - hist_p[0][3]) /
                                        max(len(hist_p) - 1, 1),
             "residual_every_5": [float(f"{x[2]:.2e}") for x in hist[4::5]],
             "planning": {k: (round(v, 3) if isinstance(v, float) else v)
                          for k, v in planning.items()}}
        if label != "fp64":
            num = sum(float(np.sum((t[a] - ref_t[a]) ** 2)) for a in t)
            den = sum(float(np.sum(ref_t[a] ** 2)) for a in t)
            r["dE_vs_fp64"] = hist[-1][1] - ref
            r["amplitude_norm_error_rel"] = math.sqrt(num / max(den, 1e-300))
            r["switched_at"] = switched
        if opts.get("learned"):
            r["fallbacks"] = fallbacks
        out[label] = r
    for label in list(runs)[1:]:
        for key, sfx in (("s_to_1uEh", ""), ("s_to_1uEh_planned", "_planned")):
            if out[label][key] and out["fp64"][key]:
                out[f"speedup_to_1uEh_{label}_vs_fp64{sfx}"] = (out["fp64"][key] /
                                                               out[label][key])
    return out


def learned_stream(local, ntrain, ntest, seed=4000):
    """the learned preconditioner on the instance stream (n_occ ~ U[6,16],
    n_virt ~ U[30,120], gap ~ U[0.2,0.8] Eh, n_aux 160, B's standard deviation
    scaled with the size so that plain diagonal + DIIS converges, see
    learned.stream): the first `ntrain`
    instances are solved with plain diagonal + DIIS (FP64) while their steps
    are sampled, the perceptron is trained on the device, and the next
    `ntest` instances are solved plain and with the learned step; iterations
    and wall time to |dE| < 1 uEh against each instance's plain converged
    energy.  Returns (report, weights)."""
    import gccu
    import learned

    insts = learned.stream(ntrain + ntest, seed, scale_sigma=True)
    rows, tg = [], []
    t0 = time.perf_counter()
    for inst in insts[:ntrain]:
        eng = gccu.Engine(local)
        try:
            smp = learned.Sampler(seed=inst["seed"])
            s = learned.solve(eng, inst, sampler=smp)
            if s.history[-1][2] < 1e-8:
                r, t = smp.targets(s)
                rows.append(r)
                tg.append(t)
        finally:
            eng.close()
    t_collect = time.perf_counter() - t0
    if not rows:
        return {"stream": f"{ntrain} training instances, seed {seed}",
                "error": "no training solve converged"}, None
    eng = gccu.Engine(local)
    try:
        t0 = time.perf_counter()
        w, l0, l1 = learned.train(eng, np.concatenate(rows), np.concatenate(tg))
        t_train = time.perf_counter() - t0
    finally:
        eng.close()
    per = []
    for inst in insts[ntrain:]:
        res = {}
        for label, weights in (("plain", None), ("learned", w)):
            eng = gccu.Engine(local)
            try:
                stamps = []
                t0 = time.perf_counter()
                s = learned.solve(eng, inst, weights=weights,
                                  callback=lambda it, en, rn: stamps.append(
                                      time.perf_counter() - t0))
                res[label] = (s.history, stamps, s.fallbacks)
            finally:
                eng.close()
        e_ref = res["plain"][0][-1][1]
        row = {"nocc": inst["nocc"], "nvirt": inst["nvir"], "gap": round(inst["gap"], 3)}
        for label, (hist, stamps, fb) in res.items():
            it = learned.iterations_to(hist, e_ref)
            row[label] = {"iterations_to_1uEh": it,
                          "s_to_1uEh": stamps[it - 1] if it else None,
                          "converged": hist[-1][2] < 1e-9}
            if label == "learned":
                row[label]["fallbacks"] = fb
                row[label]["dE_vs_plain"] = hist[-1][1] - e_ref
        per.append(row)

    def mean(label, key):
        v = [r[label][key] for r in per if r[label][key] is not None]
        return float(np.mean(v)) if v else None

    report = {
        "stream": f"{ntrain} training + {ntest} held-out instances, seed {seed}, "
                  "sigma_B = 0.035 (180/(n_occ n_virt))^(1/4)",
        "training_rows": int(sum(len(t) for t in tg)), "train_solves_converged": len(rows),
        "s_collect": t_collect, "s_train": t_train, "loss_before": l0, "loss_after": l1,
        "mean_iterations_to_1uEh": {"plain": mean("plain", "iterations_to_1uEh"),
                                    "learned": mean("learned", "iterations_to_1uEh")},
        "mean_s_to_1uEh": {"plain": mean("plain", "s_to_1uEh"),
                           "learned": mean("learned", "s_to_1uEh")},
        "fallbacks_total": int(sum(r["learned"]["fallbacks"] for r in per)),
        "held_out_not_reaching_1uEh": {
            lab: int(sum(r[lab]["iterations_to_1uEh"] is None for r in per))
            for lab in ("plain", "learned")},
        "max_abs_dE_learned_vs_plain": float(max(abs(r["learned"]["dE_vs_plain"]) for r in per)),
        "instances": per,
    }
    return report, w


def run_reference(args, cfg):
    """the oracle port of the reference path on host cores (rank 0 only)"""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    import binding
    import cc
    from engine import OracleEngine
    import hamiltonian as hm
    sp, eps, B = setup_hamiltonian(cfg)
    cores = os.cpu_count()
    binding.set_blas(cores)
    oe = OracleEngine(route=3)
    s = cc.CCSolver(oe, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
    t0 = time.time()
    from devfill import TorchIntegrals
    s.load_hamiltonian_device(TorchIntegrals(sp, eps, B, device="cpu"))
    setup_s = time.time() - t0
    seed_amplitudes(oe, s, cfg)
    stride = None
    times = []
    for i in range(1 + args.steps):
        if stride is None:
            binding.sampling(4096)
            t0 = time.time()
            s.evaluate()
            full = binding.scaled_time(time.time() - t0, binding.sampling_report())
            stride = int(max(1, min(4096, full / max(args.ref_seconds, 1e-3))))
            continue
        binding.sampling(stride)
        t0 = time.time()
        s.evaluate()
        scaled = binding.scaled_time(time.time() - t0, binding.sampling_report())
        times.append(scaled)
    binding.sampling(1)
    val = float(np.mean(times)) if times else None
    line = {
        "impl": "reference",
        "metric": metric_of(cfg),
        "value": val, "unit": "s", "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": val * 1e3 if val else None,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": data_desc(cfg) + " (same seeded Hamiltonian as the GPU arm)",
        "config": {"workload": cfg["name"], "method": "CCSD spin-orbital",
                   "nocc": cfg["nocc"], "nvirt": cfg["nvir"], "naux": cfg["naux"],
                   "sigma_B": cfg["sigma"], "use_tr": False, "setup_s": round(setup_s, 1)},
        "extrapolated": True,
        "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "port",
                         "sample": f"each step: one CCSD iteration through the oracle (route 3, "
                                   f"OpenBLAS dgemm on {cores} cores) with every {stride}-th "
                                   f"long-operand batch executed, extrapolated by batch count "
                                   f"(validated against an unsampled iteration at o12/v100 "
                                   f"with bench.py --validate-sampling)"},
        "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def seed_amplitudes(oe, s, cfg):
    """nonzero amplitudes so that no block is screened out (the reference
    skips blocks with norm^2 < 1e-28): T2 = MP2 guess -<ab||ij>/D, T1 small,
    seeded"""
    oe.add_block(1.0, s.lid("V"), 7, s.lid("R2"), 1, reset=True)
    oe.precondition(s.lid("T2"), s.lid("R2"), s.lid("DT2"), fac=-1.0)
    rng = np.random.default_rng(cfg["seed"])
    t1 = oe.data[s.lid("T1")]
    t1[:] = 1e-3 * rng.standard_normal(t1.size)


def validate_sampling(args):
    """the reference arm's extrapolation checked on a size where a full
    iteration is affordable: one unsampled oracle iteration at o12/v100 next
    to the sampled estimates at several strides"""
    import binding
    import cc
    from devfill import TorchIntegrals
    from engine import OracleEngine
    import hamiltonian as hm
    cfg = CONFIGS[10]
    sp, eps, B = setup_hamiltonian(cfg)
    cores = os.cpu_count()
    binding.set_blas(cores)
    oe = OracleEngine(route=3)
    s = cc.CCSolver(oe, hm.FactorizedIntegrals(sp, eps, B), method="ccsd")
    s.load_hamiltonian_device(TorchIntegrals(sp, eps, B, device="cpu"))
    seed_amplitudes(oe, s, cfg)
    out = {"workload": cfg["name"], "cores": cores}
    binding.sampling(1)
    t0 = time.time()
    s.evaluate()
    out["unsampled_s"] = time.time() - t0
    for stride in (4, 16, 64):
        binding.sampling(stride)
        t0 = time.time()
        s.evaluate()
        est = binding.scaled_time(time.time() - t0, binding.sampling_report())
        out[f"stride_{stride}_estimate_s"] = est
        out[f"stride_{stride}_ratio"] = est / out["unsampled_s"]
    binding.sampling(1)
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gecco-b200")
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--conv-config", type=int, default=12,
                    help="workload of the time-to-convergence comparison")
    ap.add_argument("--conv-sigma", type=float, default=None,
                    help="standard deviation of B for the convergence workload (override)")
    ap.add_argument("--conv-maxiter", type=int, default=80)
    ap.add_argument("--conv-variants", default=None,
                    help="JSON object: label -> options of CCSolver.solve_mixed, solved "
                         "after the default variants (with --only-convergence)")
    ap.add_argument("--only-convergence", action="store_true",
                    help="run only the time-to-convergence comparison and exit")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", type=int, default=3,
                    help="precision mode of the headline line: 3 (default): FP64 emulated "
                         "with four int8 slices on the tensor cores (the bulk mode of the "
                         "mixed solve), 2: five slices, 1: split TF32, 0: FP64 only; the "
                         "FP64 path and the other tensor-core modes are measured beside it")
    ap.add_argument("--no-i8", action="store_true",
                    help="skip the s/iteration of the other tensor-core precision modes")
    ap.add_argument("--no-fp64", action="store_true",
                    help="with --precision 1, skip the FP64 measurement")
    ap.add_argument("--no-use-tr", action="store_true",
                    help="skip the timing with spin-flip symmetry")
    ap.add_argument("--no-convergence", action="store_true",
                    help="skip the time-to-convergence comparisons")
    ap.add_argument("--tune", type=int, default=1,
                    help="1 (default): autotuned tile policies; 0: the fixed rule")
    ap.add_argument("--no-fixed-rule", action="store_true",
                    help="skip the fixed-rule comparison of the autotuned iteration")
    ap.add_argument("--no-d2h", action="store_true",
                    help="skip the D2h CCSD workload")
    ap.add_argument("--no-ccsdt", action="store_true",
                    help="skip the CCSDT iteration on the CCSDT configuration's workload")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned preconditioner's instance stream")
    ap.add_argument("--c4-train", type=int, default=64,
                    help="training instances of the learned preconditioner's stream (the first "
                         "64 solves of the 256-instance stream)")
    ap.add_argument("--c4-test", type=int, default=32,
                    help="held-out instances of the stream (192: the rest of the full stream)")
    ap.add_argument("--trace-contraction", default=None,
                    help="set up, run one named [CONTR] of the formula once and exit "
                         "(the command the ncu captures in profiles/ run)")
    ap.add_argument("--trace-learned", action="store_true",
                    help="set up, run the learned preconditioner step once on the doubles "
                         "lists and exit (the command the ncu captures in profiles/ run)")
    ap.add_argument("--trace-spin-prj", action="store_true",
                    help="set up, project the singlet residual of the doubles onto its "
                         "singlet part and exit (the command the ncu captures in profiles/ run)")
    ap.add_argument("--no-spin-prj", action="store_true",
                    help="skip the timing of the singlet spin projection")
    ap.add_argument("--profile-out", default=None,
                    help="write per-contraction kernel times (JSON)")
    ap.add_argument("--validate-sampling", action="store_true",
                    help="compare the reference arm's sampled estimate with an unsampled "
                         "oracle iteration at o12/v100 and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    cfg = CONFIGS[args.config]
    if args.validate_sampling:
        validate_sampling(args)
    elif args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_gpu(args, cfg)


if __name__ == "__main__":
    main()
