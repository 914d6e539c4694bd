"""Benchmark: batched river CFR+ solves/s on one or more B200s.

Workload: the batched uneven river configuration — 4,096 seeded subgames per
GPU (1-4 bet sizes from 25-200% pot, raise cap 1-3, range supports of 200-1,081
combos with lognormal(0,1) weights, pot 20-200, SPR 0.5-12), 1,000 CFR+
iterations each in FP32, then the FP64 best-response exploitability pass.
One step = one solve of the whole batch.  Each GPU solves its own batch
(weak scaling, replicas only: no data-path collective).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  `value` is device-timed with inputs resident
in HBM; `e2e` goes through the public C ABI from host buffers (pack + H2D +
solve + D2H of the results) per step.
"""
import argparse
import concurrent.futures
import importlib
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
METRIC = "batched river solves/s at <=0.1% pot exploitability vs plain kernel; evals/s"
# DRAM bytes (read + write) of one CFR iteration of the sweeps and terminals
# from a one-kernel-class-at-a-time ncu capture of a 256-subgame batch (seed 2;
# 4.5 iterations, 650.5 MB per iteration against 977.6 MB of algorithmic bytes).
# The bench scales it by the subgame count; at 256 subgames part of the round
# trips stays in L2, so the scaled figure is a lower bound.
TRAFFIC_PER_ITER = {"subgames": 256, "seed": 2, "bytes": 650.48e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--subgames", type=int, default=4096)
    ap.add_argument("--iters", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--target", type=float, default=1e-3, help="exploitability gate, fraction of the pot")
    ap.add_argument("--cpu-sample", type=int, default=0, help="subgames in the CPU baseline sample (0 = auto)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other", action="store_true", help="skip the other workloads' numbers")
    return ap.parse_args()


def max_over_ranks(x, pg, device):
    """The largest of the ranks' values of x (the job's time is its slowest
    replica's); x itself without a process group."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_seed(seed, rank):
    """Seed of a rank's own batch: replicas solve different subgames."""
    return seed + 1000 * rank


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"mtt_bench_clocks_gpu{gpu_index}_{os.getpid()}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
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


def host_cpu():
    """(CPU model, logical cores) of this host."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count() or 1


def workload_config(args, world):
    """The `config` object both arms print (identical for the same flags)."""
    return {"workload": f"batched uneven river CFR+, {args.subgames} subgames per GPU, {args.iters} alternating "
                        f"iterations + FP64 exploitability, continued to <= {args.target * 100:g}% pot",
            "subgames_per_gpu": args.subgames, "iters": args.iters, "seed": args.seed,
            "gate_pct_pot": args.target * 100,
            "l2": "inputs larger than L2 (every subgame's arrays resident: GBs per GPU)",
            "parallelism": f"replicas x{world} (weak scaling, no data-path collective)"}


def _oracle_modules():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    import pyworkload
    pyoracle.lib()
    return pyoracle, pyworkload


def cpu_oracle_sample(subs, iters, n_sample, budget_s=4.0):
    """One bounded sample of the workload on the CPU restatement of the
    reference sweeps (oracle: dense O(H^2) FP64 showdowns), all host cores:
    n_sample subgames at once, each through `it` alternating CFR+ iterations
    then the oracle's FP64 best response.  `it` is sized once so the sample
    takes about budget_s.  Returns a callable that runs one sample and gives
    (wall seconds of the sample, full-solve-equivalent seconds, it)."""
    pyoracle, _ = _oracle_modules()
    cores = os.cpu_count() or 1
    sample = subs[:n_sample]
    ex = concurrent.futures.ThreadPoolExecutor(max_workers=min(cores, len(sample)))

    def iters_part(it):
        t0 = time.perf_counter()
        outs = list(ex.map(lambda g: pyoracle.cfr_solve(g, it, alternate=1, avg_power=2.0), sample))
        return time.perf_counter() - t0, outs

    t1, _ = iters_part(1)
    it = int(max(1, min(iters, round(budget_s / max(t1, 1e-6)))))

    def one():
        ti, outs = iters_part(it)
        t0 = time.perf_counter()
        list(ex.map(lambda go: pyoracle.best_response(go[0], go[1]["S0"], go[1]["S1"]), zip(sample, outs)))
        tb = time.perf_counter() - t0
        return ti + tb, ti * (iters / it) + tb, it
    return one, min(cores, len(sample))


def run_reference(args, rank, world):
    """The CPU arm: the oracle, a restatement of the reference's kernels (the
    reference has no CPU solve path), on the host cores.  Each step is one
    bounded sample: n subgames (one per core) through a fixed number of
    alternating iterations plus the FP64 best response, sized to about 4 s.
    `ms_per_step` is the time of that sample; `value` scales it to full
    1,000-iteration solves.  The subgames come from the oracle's own
    restatement of the workload generator, so the product library is never
    loaded."""
    if rank != 0:
        return
    _, pyworkload = _oracle_modules()
    n_sample = args.cpu_sample or max(os.cpu_count() or 1, 8)
    subs = pyworkload.river_batch(n=n_sample, seed=args.seed)
    one, threads = cpu_oracle_sample(subs, args.iters, n_sample)
    for _ in range(args.warmup):
        one()
    wall, equiv, it = 0.0, 0.0, 1
    for _ in range(args.steps):
        w, e, it = one()
        wall += w
        equiv += e
    steps = max(args.steps, 1)
    v = n_sample * steps / equiv if equiv > 0 else 0.0
    model, ncpu = host_cpu()
    sample = (f"{n_sample} of the {args.subgames} subgames (seed {args.seed}) per step, each through {it} of "
              f"{args.iters} alternating CFR+ iterations (dense O(H^2) FP64 showdowns) + the FP64 best response, "
              f"{threads} threads; scaled to {args.iters}-iteration solves (the per-iteration cost does not depend "
              f"on t); the gate continuation of the subgames above {args.target * 100:g}% pot is not sampled")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded)", "config": workload_config(args, world),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample,
                             "cpu_model": model, "nproc": ncpu},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_kernels_leg(mtt, wl, stream, iters):
    """The reference's own heads-up sweep kernels (oracle/_ref/ref_hu_sweeps,
    built from honest_multistreet_solver.cu:88-249) against this build's
    kernels on the same river subgame: 1,024 of the board's live combos for
    both players, uniform ranges, pot 100, stack 200, a 75% bet plus all-in and
    one raise (the reference holds three actions per node), `iters` CFR+
    iterations with simultaneous updates and linear averaging in the
    reference semantics, no best response.  Both timed with CUDA events after
    a warm-up."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyref
    if not pyref.available():
        return {"unavailable": "oracle/_ref/ref_hu_sweeps not built (make -C oracle ref REF=<reference checkout>)"}
    sub = wl.river_uniform(seed=0, n_hands=1024, bet_sizes=(0.75,))
    try:
        ref_ms, launches = pyref.run(sub, iters, timing=True)[4:]
    except Exception as e:   # the harness refuses inputs it cannot index safely
        return {"unavailable": f"reference harness: {e}"}
    b = mtt.RiverBatch([sub])
    p = mtt.solve_params(iters=iters, algo=0, semantics=1, alternate=False, avg_power=1.0, exploitability=False)
    out = {"workload": f"river, 1,024 live combos per player, uniform ranges, pot 100, stack 200, 75% bet + all-in, "
                       f"1 raise, {iters} CFR+ iterations (simultaneous, linear averaging, reference semantics), "
                       f"no best response", "reference_ms": ref_ms, "reference_launches": launches}
    for name, graph in (("plain_ms", False), ("graph_ms", True)):
        b.solve(p, graph=graph)
        out[name] = _event_ms(lambda: b.solve(p, graph=graph), stream)
    b.close()
    out["vs_reference_kernels"] = ref_ms / out["graph_ms"]
    out["vs_reference_kernels_plain"] = ref_ms / out["plain_ms"]
    return out


def _event_ms(fn, stream, reps=1):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def other_configs(mtt, wl, stream):
    """Device-timed numbers of the other workloads (one run each, after a
    warm-up run): the single river subgame, the turn+river DCFR solve, the
    differentiable EV over 1,024 boards, the four-player ICM river, the leaf
    network's GEMM and training step, the preflop chain, the full flop-EV
    dump, the flop-subset selection, the flop subgame and the depth-limited
    turn solve."""
    import torch
    out = {}
    # single river subgame, uniform ranges, 1,000 CFR+ iterations + FP64 exploitability
    sub = wl.river_uniform(seed=0)
    b = mtt.RiverBatch([sub])
    p0 = mtt.solve_params(iters=1000, threads=0, avg_power=2.0)
    p0.threads = b.autotune(p0)        # the library's schedule search (untimed)
    b.solve(p0, graph=True)
    t = _event_ms(lambda: b.solve(p0, graph=True), stream)
    out["river_single"] = {"ms": t, "exploitability_pct_pot": float(b.results()[0, 5] * 100),
                           "workload": "river, uniform 1,081-combo ranges, pot 100, stack 200, bets 50/100% + all-in, "
                                       "1 raise, 1,000 alternating CFR+ iterations + FP64 best response"}
    b.close()
    # turn + river DCFR
    sub = wl.turn_dcfr(seed=1)
    b = mtt.RiverBatch([sub])
    p1 = mtt.solve_params(iters=500, algo=mtt.ALGO_DCFR, alpha=1.5, beta=0.0, gamma=2.0, threads=0)
    p1.threads = b.autotune(p1)
    b.solve(mtt.solve_params(iters=5, algo=mtt.ALGO_DCFR, threads=p1.threads), graph=True)
    t = _event_ms(lambda: b.solve(p1, graph=True), stream)
    out["turn_river_dcfr"] = {"ms": t, "exploitability_pct_pot": float(b.results()[0, 5] * 100),
                              "nodes": int(len(sub["nodes"])), "iter_bytes": b.info()["iter_bytes"],
                              "workload": "turn board, 48 rivers, Dirichlet(0.3) ranges (1,128 live combos), pot 60, "
                                          "stack 470, bets 33/75/150% + all-in, 2 raises, DCFR(1.5, 0, 2) x 500"}
    b.close()
    # differentiable EV of softmax strategies
    dv = importlib.import_module("mtt-gpu-solver_b200.diffev")
    subs, logits = wl.diff_boards(n=1024, seed=3)
    sev = dv.StrategyEV(subs)
    L = torch.randn(sev.total_rows, device="cuda")
    R = torch.zeros(sev.total_range, device="cuda")
    for s_, g in enumerate(subs):
        o = int(sev.range_off[s_]); H = len(g["combos0"]); Hp = (H + 3) // 4 * 4
        R[o:o + H] = torch.from_numpy(g["range0"]).to("cuda")
        R[o + Hp:o + Hp + H] = torch.from_numpy(g["range1"]).to("cuda")
    sev.batch.ev_grad(L, R)
    t = _event_ms(lambda: sev.batch.ev_grad(L, R), stream)
    out["diff_ev"] = {"ms": t, "boards_per_s": 1024 / (t * 1e-3),
                      "workload": "1,024 river boards, config-0 trees, N(0,1) logits: root EV + adjoint (range and "
                                  "logit gradients)"}
    sev.close()
    # four-player ICM river
    mw = importlib.import_module("mtt-gpu-solver_b200.multiway")
    sub = wl.multiway_icm(seed=4)
    mb = mw.MultiwayBatch([sub])
    p4 = mtt.solve_params(iters=200)
    mb.solve(p4, graph=True)
    t = _event_ms(lambda: mb.solve(p4, graph=True), stream)
    out["multiway_icm"] = {"ms": t, "nodes": int(len(sub["nodes"])), "values": mb.values()[0].tolist(),
                           "workload": "4 players, 1,081 combos, Dirichlet(0.3) ranges, Malmuth-Harville bubble "
                                       "factors (50/30/20 over 8 seats), bets 50/100% + a pot-sized raise re-raised "
                                       "up to twice, 200 CFR+ iterations, card removal against the hero's hand and "
                                       "split ties (correct semantics)"}
    mb.close()
    # leaf network: one GEMM of the first layer and one training step of 4,096 samples
    ln = importlib.import_module("mtt-gpu-solver_b200.leafnet")
    gt = ln.gemm_timing(4096, 1024, 2752, reps=20)
    out["leaf_gemm"] = {"ms": gt["graph_ms"], "tflops": gt["graph_tflops"], "shape": [4096, 1024, 2752],
                        "per_call_ms": gt["call_ms"], "per_call_tflops": gt["call_tflops"],
                        "timing": "20 launches captured in one CUDA graph and replayed (ms per launch); per_call: "
                                  "20 Python calls, host work between launches included"}
    net = ln.LeafNet(batch_cap=4096, seed=0)
    X = torch.randn(4096, 2706, device="cuda") * 0.5
    T = torch.randn(4096, 2652, device="cuda") * 0.3
    net.train_step(X, T, lr=1e-4, want_loss=False)
    t = _event_ms(lambda: net.train_step(X, T, lr=1e-4, want_loss=False), stream, reps=5)
    out["leaf_train_step"] = {"ms": t, "samples_per_s": 4096 / (t * 1e-3),
                              "tflops": 3 * 15.17e6 * 4096 / (t * 1e-3) / 1e12,
                              "workload": "4,096 samples, 2,706 -> 3 x 1,024 -> 2,652, BF16 tcgen05 GEMMs + Adam"}
    net.close()
    # preflop chain
    pf = importlib.import_module("mtt-gpu-solver_b200.preflop")
    flops, w = pf.read_subset(os.path.join(ROOT, "tests", "golden", "mtt_subset.bin"))

    def chain():
        allin = pf.allin_matrix(pf.REFERENCE)
        mats = pf.flop_class_matrices(flops, pf.REFERENCE)
        pf.dcfr(w, mats, allin, iters=500)
    chain()
    out["preflop_chain"] = {"ms": _event_ms(chain, stream),
                            "workload": "169x169 all-in matrix (3,000 samples/pair) + 100 class-reduced flop matrices "
                                        "+ 500 DCFR iterations (reference mode)"}
    # full flop-EV dump
    f4 = torch.from_numpy(np.ascontiguousarray(mtt.canonical_flops()[:, :3])).to("cuda")
    mtt.ev_dump(f4[:8])
    out["ev_dump_1755"] = {"ms": _event_ms(lambda: mtt.ev_dump(f4), stream),
                           "workload": "all 1,755 canonical flops, reference runout subsample (bit-exact dump)"}
    # flop subset by NN-OMP over the regenerated dump
    subset = importlib.import_module("mtt-gpu-solver_b200.subset")
    cols = mtt.ev_dump(f4).reshape(1755, -1)
    colw = mtt.canonical_flops()[:, 3].astype(np.float64)
    subset.nnomp(cols, colw, 100)
    out["flop_subset_nnomp"] = {"ms": _event_ms(lambda: subset.nnomp(cols, colw, 100), stream),
                                "workload": "optimize_subset.py on the device: 100 greedy NN-OMP steps over the "
                                            "1,755 x 1,352 dump (resident), FP64 Lawson-Hanson refits; one "
                                            "mtt_subset_nnomp call including its weight upload and result read-back"}
    # flop subgame: flop and turn betting, 49 turn cards, river run out
    sub = wl.flop_runout(seed=9)
    b = mtt.RiverBatch([sub])
    pf3 = mtt.solve_params(iters=300, alternate=True, avg_power=2.0)
    pf3.threads = b.autotune(pf3)
    b.solve(pf3, graph=True)
    t = _event_ms(lambda: b.solve(pf3, graph=True), stream)
    out["flop_turn_runout"] = {"ms": t, "exploitability_pct_pot": float(b.results()[0, 5] * 100),
                               "nodes": int(len(sub["nodes"])), "iter_bytes": int(b.info()["iter_bytes"]),
                               "workload": "flop board, Dirichlet(0.3) ranges (1,176 live combos), pot 100, stack 150, "
                                           "bets 50/100% + all-in, 1 raise on flop and turn, 49 turn cards then the "
                                           "river run out (2,402 table variants), 300 alternating CFR+ iterations "
                                           "+ FP64 best response"}
    b.close()
    # depth-limited turn solve: leaf network trained on leaf samples of 64 full solves
    dlm = importlib.import_module("mtt-gpu-solver_b200.depthlimit")
    t0 = time.perf_counter()
    X, T, W, meta = dlm.leaf_training_set(64, seed=100, iters=300)
    net = dlm.train_on(X, T, W, meta, epochs=3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    spot = dlm.turn_spot(seed=0)
    res, ms = {}, {}
    for name, kw in (("full", {"limited": False}), ("net", {"limited": True, "net": net}),
                     ("checkdown", {"limited": True, "net": None})):
        dlm.solve(spot, iters=20, **kw)
        ms[name] = _event_ms(lambda: res.__setitem__(name, dlm.solve(spot, iters=300, **kw)), stream, reps=1)
    leaf = [dlm.leaf_errors_in_situ(dlm.turn_spot(seed=s), net, iters=300) for s in (0, 1, 2)]
    out["depth_limited_turn"] = {
        "solve_ms": {k: v for k, v in ms.items()},
        "solve_ms_note": "one depthlimit.solve call: tree and table packing, upload, 300 iterations, read-back",
        "root_value_error_pot": {k: dlm.errors(spot, res[k], res["full"])["value"] for k in ("net", "checkdown")},
        "leaf_mae_pot": {k: float(np.mean([e[k] for e in leaf])) for k in ("net", "checkdown")},
        "train_s": train_s, "train_samples": int(len(X)),
        "workload": "turn spot pot 100, stack 150, bets 50/100% + all-in, 1 raise, Dirichlet(0.3) ranges (1,128 "
                    "combos), 300 alternating CFR+ iterations: full turn + river tree vs 5 depth-limit leaves valued "
                    "by check-down (fixed-point scans) or check-down + leaf network; leaf MAE measured at 3 held-out "
                    "spots' leaves against their full solve"}
    net.close()
    return out


def run_b200(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    mtt = importlib.import_module("mtt-gpu-solver_b200")
    wl = importlib.import_module("mtt-gpu-solver_b200.workloads")
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    subs = wl.river_batch(n=args.subgames, seed=replica_seed(args.seed, rank))
    # 1,000 alternating CFR+ iterations per subgame, then the FP64 best
    # response; subgames still above 0.1% of the pot continue in chunks of 250
    # iterations (compacted work lists) until they pass, up to 4x the budget.
    # (Chunks of 500 / 250 / 125 / 50 measured 299 / 256 / 299 / 466 ms of
    # continuation at 4,096 subgames, seed 2: a shorter chunk stops the passing
    # subgames sooner but adds a best response and a compaction per chunk.)
    p = mtt.solve_params(iters=args.iters, threads=0, exploitability=True, alternate=True, avg_power=2.0,
                         target_expl=args.target, max_iters=4 * args.iters, chunk_iters=max(args.iters // 4, 1))
    stream = torch.cuda.current_stream()
    batch = mtt.RiverBatch(subs)
    threads = batch.autotune(p)
    p.threads = threads
    sched = batch.schedule()       # autotuned: CTA size, hands per warp item, terminals per CTA
    info = batch.info()

    def step():
        batch.solve(p, graph=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    launches0 = batch.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_launches = batch.launch_count() - launches0
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    ms = max_over_ranks(ms, pg, "cuda")
    res = batch.results()
    expl = res[:, 5]
    its = batch.iterations()
    # the same solve with the iteration count fixed at --iters (no gate)
    pf = mtt.solve_params(iters=args.iters, threads=threads, exploitability=True, alternate=True, avg_power=2.0)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    batch.solve(pf, graph=True)
    f1.record(stream)
    torch.cuda.synchronize()
    fixed_ms = f0.elapsed_time(f1)
    fixed_expl = batch.results()[:, 5]
    # the sweeps and terminals alone (no best response): algorithmic bytes / event time
    ps = mtt.solve_params(iters=args.iters, threads=threads, exploitability=False, alternate=True, avg_power=2.0)
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    batch.solve(ps, graph=True)
    k0.record(stream)
    batch.solve(ps, graph=True)
    k1.record(stream)
    torch.cuda.synchronize()
    solve_ms = k0.elapsed_time(k1)
    algo_bytes = info["iter_bytes"] * args.iters
    achieved = algo_bytes / (solve_ms * 1e-3) / 1e9
    traffic = (TRAFFIC_PER_ITER["bytes"] * args.subgames / TRAFFIC_PER_ITER["subgames"]
               if args.seed == TRAFFIC_PER_ITER["seed"] else None)
    peak, peak_kind = load_peaks()
    # per kernel class: CUDA events around each class in every pass (level
    # launches without the graph), compulsory bytes from the work lists
    kp = batch.kernel_profile(ps, iters=min(args.iters, 10))
    kernels = {}
    for k, v in kp.items():
        gbs = v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] > 0 else 0.0
        kernels[k] = {"ms_per_iter": v["ms"], "compulsory_bytes_per_iter": int(v["bytes"]), "gbs": gbs,
                      "frac": gbs / peak}
    sw_b = kp["k_fwd"]["bytes"] + kp["k_bwd"]["bytes"]
    sw_ms = kp["k_fwd"]["ms"] + kp["k_bwd"]["ms"]
    kernels["sweeps"] = {"kernels": "k_fwd + k_bwd", "gbs": sw_b / (sw_ms * 1e-3) / 1e9,
                         "frac": sw_b / (sw_ms * 1e-3) / 1e9 / peak}
    batch.close()

    # end to end through the public API from host buffers.  A step is one batch:
    # create (pack on host threads, allocate, upload), solve, results (device ->
    # host) and close.  Steps are double-buffered as a serving loop runs them:
    # the next step's batch is created on a host thread while the current one
    # solves on its own non-blocking stream.  The first step's creation is not
    # hidden and is inside the timed region.
    e2e_parts = {"create": 0.0, "solve": 0.0, "results": 0.0, "close": 0.0}
    e2e_stream = torch.cuda.Stream()
    dev = torch.cuda.current_device()

    def make_batch():
        torch.cuda.set_device(dev)                # a new host thread starts on device 0
        t = time.perf_counter()
        b = mtt.RiverBatch(subs)
        return b, time.perf_counter() - t

    def e2e_run(n):
        with concurrent.futures.ThreadPoolExecutor(1) as ex:
            nxt = ex.submit(make_batch)
            for k in range(n):
                b, tc = nxt.result()
                e2e_parts["create"] += tc
                if k + 1 < n:
                    nxt = ex.submit(make_batch)
                t = [time.perf_counter()]
                b.solve(p, stream=e2e_stream, graph=True)
                t.append(time.perf_counter())
                b.results(stream=e2e_stream)      # synchronises
                t.append(time.perf_counter())
                b.close()
                t.append(time.perf_counter())
                for i, name in enumerate(("solve", "results", "close")):
                    e2e_parts[name] += t[i + 1] - t[i]
    e2e_run(1)
    torch.cuda.synchronize()
    for k in e2e_parts:
        e2e_parts[k] = 0.0
    t0 = time.perf_counter()
    n_e2e = max(1, min(args.steps, 3))
    e2e_run(n_e2e)
    e2e_s = (time.perf_counter() - t0) / n_e2e
    e2e_s = max_over_ranks(e2e_s, pg, "cuda")
    h2d = sum(g["nodes"].nbytes + g["combos0"].nbytes + g["combos1"].nbytes + g["range0"].nbytes +
              g["range1"].nbytes for g in subs)

    # the plain single-instance kernel: the same solve (same parameters, gate
    # included) on one subgame at a time, launched level by level with no
    # batching and no graph; inputs resident, CUDA events around the solves only
    n_plain = min(8, len(subs))
    singles = [mtt.RiverBatch([g]) for g in subs[:n_plain]]
    singles[0].solve(p)
    torch.cuda.synchronize()
    plain_ms = _event_ms(lambda: [b1.solve(p) for b1 in singles], stream)
    for b1 in singles:
        b1.close()
    plain_value = n_plain / (plain_ms * 1e-3)

    ref_kernels = reference_kernels_leg(mtt, wl, stream, args.iters) if not args.no_other else None

    # evaluator throughput (all C(52,7) hands)
    mtt.eval7_enumerate()
    torch.cuda.synchronize()
    v0 = torch.cuda.Event(enable_timing=True)
    v1 = torch.cuda.Event(enable_timing=True)
    v0.record(stream)
    for _ in range(5):
        mtt.eval7_enumerate()
    v1.record(stream)
    torch.cuda.synchronize()
    evals_per_s = 5 * 133784560 / (v0.elapsed_time(v1) * 1e-3)

    other = {} if args.no_other else other_configs(mtt, wl, stream)

    value = args.subgames * world / (ms * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded)",
            "config": workload_config(args, world),
            "launch": {"cta_threads": threads, "schedule": sched, "resident_bytes": int(info["device_bytes"])},
            "exploitability_pct_pot": {"median": float(np.median(expl) * 100), "max": float(np.max(expl) * 100),
                                       "frac_le_gate": float(np.mean(expl <= args.target)),
                                       "gate": args.target * 100},
            "iterations": {"mean": float(np.mean(its)), "max": int(np.max(its)),
                           "frac_continued": float(np.mean(its > args.iters))},
            "fixed_iters": {"iters": args.iters, "solves_per_s": args.subgames * world / (fixed_ms * 1e-3),
                            "frac_le_gate": float(np.mean(fixed_expl <= args.target)),
                            "max_expl_pct_pot": float(np.max(fixed_expl) * 100)},
            "evals_per_s": evals_per_s,
            "plain_kernel": {"value": plain_value, "unit": "solves/s", "ms": plain_ms,
                             "sample": f"{n_plain} subgames solved one at a time (same parameters and gate), level "
                                       f"launches, no graph; CUDA events around the solves, inputs resident"},
            "vs_plain": value / plain_value,
            "reference_kernels": ref_kernels,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_unit": "DRAM bytes per CFR iteration: ncu capture of a 256-subgame batch scaled "
                                         "by the subgame count (a lower bound: part of the small batch's round "
                                         "trips stays in L2)",
                         "algorithmic_bytes_per_iter": int(info["iter_bytes"]),
                         "kernel": "CFR sweeps + terminals (k_fwd, k_term, k_bwd), no best response",
                         "peak_kind": peak_kind, "kernel_ms": solve_ms, "per_kernel": kernels},
            "clocks": clocks,
            "e2e": {"value": args.subgames * world / e2e_s, "unit": "solves/s",
                    "host_s_per_step": {k: v / n_e2e for k, v in e2e_parts.items()},
                    "pipeline": "double-buffered: each next batch is created on a host thread while the "
                                "current one solves; host_s_per_step.create overlaps the solve",
                    "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(args.subgames * 6 * 8)},
            "gpu_launches": int(gpu_launches),
            "other_configs": other}
    if rank == 0 and not args.no_cpu_baseline:
        _, pyworkload = _oracle_modules()
        n_sample = args.cpu_sample or max(os.cpu_count() or 1, 8)
        one, threads_cpu = cpu_oracle_sample(pyworkload.river_batch(n=n_sample, seed=args.seed), args.iters,
                                             n_sample, budget_s=8.0)
        wall, equiv, it = one()
        model, ncpu = host_cpu()
        line["cpu_baseline"] = {"value": n_sample / equiv, "unit": "solves/s", "cores": threads_cpu, "kind": "port",
                                "sample": f"{n_sample} subgames x {it} of {args.iters} alternating CFR+ iterations "
                                          f"(dense O(H^2) FP64 showdowns) + FP64 best response, {threads_cpu} "
                                          f"threads, {wall:.1f} s; scaled to full solves",
                                "cpu_model": model, "nproc": ncpu}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
