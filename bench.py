"""Benchmark: one GA generation (evaluate, select, breed, mutate) per step on the B200.

Workload: population 4,096 on a 64x64 toroidal grid, 4,739 synthetic catalog words all active, 256
secrets per cell drawn from a 2,315-word secret subset (3 episodes per secret), radius-1 rank selection,
reference crossover temperatures, mutation p = 0.05, sigma = 0.02. Genomes are the reference's FP16
layout (bootstrap He-normal weights, N(0, 0.05) tails).

The headline form (default --form tc-trunk-fp16) runs encoder, trunk and scoring on tcgen05 with FP16
operands and a top-2 margin guard (--tau, default 1e-3 x the score scale) that sends uncertain game steps
through the exact FP32 path. The plain FP32 form is timed on the same workload in the same process and
reported beside it ("plain_fp32"), with the guess agreement and fitness delta of the headline form against it over the
whole population ("agreement_with_plain"). --form fp32 benchmarks the plain form alone.

On the full workload at N=1 the line also carries "surrogate_vs_plain": the plain FP32 form evolves 50
generations and its held-out mean solve rate becomes the target; the learned-surrogate method then evolves
from the same start until it reaches that rate, and the two wall times are reported (--no-surrogate skips it).

Prints one JSON line (rank 0). `--impl reference` times the reference's own CPU path (its host-callable
model, scoring and Wordle code composed into its episode loop, built in oracle/_ref) on a bounded sample
of the same workload with every host thread.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MEASURED = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "eval_fp32_traffic.json"
TRAFFIC_TCT = ROOT / "profiles" / "eval_tct_traffic.json"
KERNELS_PER_GENERATION = 7  # prepare, evaluate, finalize, summarize, select, plan slots, breed
FORMS = {"fp32": 0, "tc-bf16": 1, "tc-fp16": 2, "tc-trunk-bf16": 3, "tc-trunk-fp16": 4}
FORM_NAMES = {"fp32": "plain fp32", "tc-bf16": "tensor-core bf16 scoring, exact fp32 re-scoring",
              "tc-fp16": "tensor-core fp16 scoring, exact fp32 re-scoring",
              "tc-trunk-bf16": "tensor-core bf16 encoder+trunk+scoring, margin guard tau with exact fp32 fallback",
              "tc-trunk-fp16": "tensor-core fp16 encoder+trunk+scoring, margin guard tau with exact fp32 fallback"}
EXTRA_KERNELS = {"fp32": 0, "tc-bf16": 1, "tc-fp16": 1, "tc-trunk-bf16": 2, "tc-trunk-fp16": 2}
DTYPES = {"fp32": "fp32 (fp16-stored genomes)",
          "tc-bf16": "bf16 tensor-core scores, fp32 trunk and exact fp32 re-scoring",
          "tc-fp16": "fp16 tensor-core scores, fp32 trunk and exact fp32 re-scoring",
          "tc-trunk-bf16": "bf16 tensor-core operands, fp32 accumulation; exact fp32 path for guarded steps",
          "tc-trunk-fp16": "fp16 tensor-core operands, fp32 accumulation; exact fp32 path for guarded steps"}


def algorithmic_flops(steps: int, encoded: int, action_count: int) -> float:
    """2 * (9,472 per encoded turn + (123,136 + 64 A) per game step): encoder 10 gathered columns x 128 +
    128 x 64; trunk 321x256 + 256x128 + 128x64; scoring 64 per action."""
    return 2.0 * (9472.0 * encoded + (123136.0 + 64.0 * action_count) * steps)


def peaks() -> dict:
    if MEASURED.exists():
        m = json.loads(MEASURED.read_text())
        return dict(hbm_gbs=m["hbm_gbs"], bf16_tflops=m["bf16_tflops"], sm_max_mhz=m.get("sm_max_mhz", 1965.0),
                    source="measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, sm_max_mhz=1965.0, source="fallback")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(gpus: int):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _all_reduce(value: float, world: int, op_name: str) -> float:
    """One FP64 all-reduce over the ranks (a device tensor under NCCL, a host tensor under gloo)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, world: int) -> float:
    """The slowest rank's time: every multi-GPU number is timed as the maximum over ranks."""
    return _all_reduce(value, world, "MAX")


def sum_over_ranks(value: float, world: int) -> float:
    """Work summed over ranks (each rank evolves its own population: weak scaling)."""
    return _all_reduce(value, world, "SUM")


def cpu_reference_rate(catalog, offsets, words, genomes_u16, action_count, sample_individuals, threads):
    """game-steps/s of the reference's CPU path on `sample_individuals` genomes (oracle/_ref/libref_host.so)."""
    from oracle import pyoracle as O

    if O.ref_host() is None:
        return None
    n = len(genomes_u16)
    cells = np.arange(n, dtype=np.uint32)
    t0 = time.perf_counter()
    raw, steps, status = O.ref_host_evaluate(genomes_u16, action_count, catalog, offsets[:n + 1], words, cells,
                                             threads)
    dt = time.perf_counter() - t0
    assert (status == 0).all()
    return float(steps.sum()) / dt, dt, int(steps.sum())


def time_generations(rt, torch, stream, world, local, steps_count, gen, counts, cfg, sample_clocks=False):
    """Times `steps_count` generations (barrier + synchronize on both sides, CUDA events on the runtime's stream)."""
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    agg = {"steps": 0, "encoded": 0, "kernel_ms": [], "rescored": 0, "full": 0, "candidates": 0, "fallbacks": 0}
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local) if sample_clocks else None
    if clocks is not None:
        clocks.__enter__()
    start.record(stream)
    for _ in range(steps_count):
        rt.advance(seed=1000 + gen, counts=counts, config=cfg)
        st = rt.stats()
        agg["steps"] += st.game_steps
        agg["encoded"] += st.encoded_turns
        agg["kernel_ms"].append(st.eval_kernel_ms)
        agg["rescored"] += st.rescored_chunks
        agg["full"] += st.full_rescores
        agg["candidates"] += st.candidate_chunks
        agg["fallbacks"] += st.fallback_steps
        gen += 1
    end.record(stream)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.__exit__(None, None, None)
    barrier(world)
    agg["ms"] = max_over_ranks(start.elapsed_time(end), world)
    agg["clocks"] = clocks.summary() if clocks is not None else None
    return agg, gen


def agreement_sample(rt, torch, counts, form, tau, episodes):
    """Guess agreement and fitness delta of `form` against the plain form on the current generation.

    A game step counts as comparable while every earlier choice of the game agreed in both runs."""
    p = rt.population
    out = {}
    for f in (0, form):
        rt.set_form(f)
        if f != 0:
            rt.set_margin_guard(tau)
        choices = torch.full((p, episodes, 6), -1, dtype=torch.int32, device="cuda")
        rt.evaluate_traced(counts, episodes, choices.data_ptr())
        torch.cuda.synchronize()
        out[f] = (choices.cpu().numpy(), rt.current_generation()["fitness"].copy())
    a, b = out[form][0], out[0][0]
    valid = (a >= 0) | (b >= 0)
    differ = a != b
    ok = valid & ~differ
    cont = np.concatenate([np.ones(a.shape[:2] + (1,), bool), np.cumprod(ok, axis=2)[:, :, :-1].astype(bool)], 2)
    total = int((cont & valid).sum())
    same = int((cont & ok).sum())
    dfit = np.abs(out[form][1].astype(np.float64) - out[0][1].astype(np.float64))
    return {"identical_guess_fraction": same / max(total, 1), "comparable_game_steps": total,
            "games": int(valid[:, :, 0].sum()), "fitness_delta_max": float(dfit.max()),
            "fitness_delta_mean": float(dfit.mean()),
            "individuals_with_changed_fitness": int((dfit > 0).sum())}


def surrogate_vs_plain(nwg, wl, torch, generations: int, min_generations: int = 8) -> dict:
    """The learned-surrogate method against the plain FP32 form at equal fitness, on this workload's grid.

    The plain form evolves `generations` generations (prepare + assemble, timed with device syncs); its population's
    mean solve rate on held-out secrets (the same cells, a second seeded draw of 256 secrets each, untimed) is the
    target. The surrogate method (4 candidates per cell, network screening with a Spearman audit and full-evaluation
    fallback, children played with the FP16 tensor-core trunk form) then evolves from the same generation 0 until its
    held-out solve rate reaches the target (and for at least `min_generations`, so the trace shows whether the rate
    holds), or for `generations` generations; its time is the steps' own clocks up to the first crossing.
    Both are measured on held-out secrets so that keeping the best-measured child (winner's curse) does not count.
    """
    capi, W = nwg.capi, nwg.workload
    train = wl.cell_lists()
    held = W.fixed_cell_lists(wl.population, wl.secrets_per_cell,
                              W.secret_subset(wl.action_count, wl.secret_subset, wl.seed), wl.seed + 101)
    counts = capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    catalog = wl.catalog()

    def population(form):
        rt = nwg.Runtime(wl.action_count, wl.population, wl.columns)
        rt.set_form(form)
        if form >= 3:
            rt.set_margin_guard(1e-3)
        rt.bootstrap(wl.population, seed=7)
        rt.set_cell_words(*train)
        return rt

    def heldout(rt):
        rt.set_cell_words(*held)
        rt.evaluate(counts)
        rate = rt.solve_rates()[1]
        rt.set_cell_words(*train)
        rt.evaluate(counts)  # the training fitness again (deterministic), for the next selection
        return rate

    rt = population(0)
    # how reliable one measured fitness is: the same population on the training and on the held-out secrets
    rt.evaluate(counts)
    f_train = rt.current_generation()["fitness"].copy()
    start = heldout(rt)
    rt.set_cell_words(*held)
    rt.evaluate(counts)
    f_held = rt.current_generation()["fitness"].copy()
    rt.set_cell_words(*train)
    rt.evaluate(counts)
    rank = lambda v: np.argsort(np.argsort(v, kind="stable"), kind="stable").astype(np.float64)
    retest = float(np.corrcoef(rank(f_train), rank(f_held))[0, 1])
    plain_s = 0.0
    for g in range(generations):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rt.prepare(5000 + g, counts, config=cfg)
        rt.assemble()
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
    target = heldout(rt)
    rt.close()

    rt = population(4)
    # Fitness measured on 768 games per individual has a test-retest rank correlation near 0.06 at this workload,
    # which caps any predictor's audit Spearman against measured fitness near its square root (about 0.25); the
    # audit floor is therefore 0 here (screen while the network's ranks agree with measurement at all).
    sc = capi.SurrogateConfig(seed=1, spearman_floor=0.0, train_steps=32)
    sur = capi.Surrogate(rt, catalog, sc,
                         secret_pool=W.secret_subset(wl.action_count, wl.secret_subset, wl.seed))
    sur_s, reached, rows = 0.0, None, []
    screened = 0
    last = None
    for g in range(generations):
        st = sur.advance(9000 + g, counts, cfg)
        sur_s += st.ms_total * 1e-3
        screened += int(st.screened)
        rate = heldout(rt)
        last = st
        rows.append({"generation": int(st.generation), "seconds": round(sur_s, 3), "heldout_solve_rate": rate,
                     "screened": bool(st.screened), "audit_spearman": None if st.spearman != st.spearman
                     else round(float(st.spearman), 4),
                     "model_pick_over_plain_child": None if st.mean_fitness_model_pick != st.mean_fitness_model_pick
                     else round(st.mean_fitness_model_pick / st.mean_fitness_first_candidate, 4)})
        if reached is None and rate >= target:
            reached = (int(st.generation), sur_s)
        if reached is not None and len(rows) >= min_generations:
            break
    sur.close()
    rt.close()
    return {
        "target": f"plain FP32 form's held-out mean solve rate after {generations} generations",
        "plain": {"generations": generations, "seconds": plain_s, "generations_per_s": generations / plain_s,
                  "heldout_solve_rate_start": start, "heldout_solve_rate_end": target},
        "surrogate": {"generations_to_target": reached[0] if reached else None,
                      "seconds_to_target": reached[1] if reached else None, "seconds_run": sur_s,
                      "generations_per_s": len(rows) / sur_s, "screened_steps": screened,
                      "last_step_ms": {k: round(getattr(last, k), 2) for k in
                                       ("ms_select_breed", "ms_descriptors", "ms_inference", "ms_evaluation",
                                        "ms_training", "ms_install", "ms_total")},
                      "trace": rows},
        "time_ratio": (reached[1] / plain_s) if reached else None,
        "fitness_test_retest_spearman": retest,
        "method": "4 candidates per cell, MLP 8192-512-128-1 on 128 probe-state descriptors (32 Adam steps per "
                  "generation), the best-scored candidate of each cell played plus a 5% audit sample, full evaluation of every candidate while the network is "
                  "untrained or the audit Spearman < 0; FP16 tensor-core trunk form",
    }


def run_ours(args) -> None:
    import torch

    rank, world, local = dist_setup(args.gpus)
    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    wl = {"full": nwg.workload.FULL, "medium": nwg.workload.MEDIUM, "small": nwg.workload.SMALL}[args.workload]
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    nwg.capi.upload_catalog(catalog)
    stream = torch.cuda.current_stream()
    rt = nwg.Runtime(wl.action_count, wl.population, wl.columns, stream=stream.cuda_stream)
    rt.set_cell_words(offsets, words)
    trunk_form = args.form.startswith("tc-trunk")
    rt.set_form(FORMS[args.form])
    if trunk_form:
        rt.set_margin_guard(args.tau)
    rt.bootstrap(wl.population, seed=0 + rank)
    counts = nwg.capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = nwg.capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)

    # CPU baseline sample: the reference CPU path on the first genomes of generation 0 (rank 0, N=1 only).
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = min(wl.population, max(2, threads))
        genomes = np.stack([rt.download_slot(i).view(np.uint16) for i in range(sample)])
        res = cpu_reference_rate(catalog, offsets, words, genomes, wl.action_count, sample, threads)
        if res is not None:
            rate, dt, steps = res
            cpu = {"value": rate, "unit": "game-steps/s", "cores": threads, "kind": "reference",
                   "sample": f"generation-0 evaluation of {sample} of {wl.population} individuals "
                             f"({steps} game steps, {dt:.1f} s) with {threads} threads"}

    gen = 0
    for _ in range(args.warmup):
        rt.advance(seed=1000 + gen, counts=counts, config=cfg)
        gen += 1

    # ---- device-resident timed region ----
    agg, gen = time_generations(rt, torch, stream, world, local, args.steps, gen, counts, cfg, sample_clocks=True)
    ms = agg["ms"]
    steps = agg["steps"]
    total_steps = sum_over_ranks(float(steps), world)

    # ---- end-to-end through the public API with host buffers ----
    pinned_offsets = torch.from_numpy(offsets).pin_memory().numpy()
    pinned_words = torch.from_numpy(words).pin_memory().numpy()
    e2e_start = torch.cuda.Event(enable_timing=True)
    e2e_end = torch.cuda.Event(enable_timing=True)
    e2e_steps = 0
    e2e_iters = max(1, min(args.steps, 3))
    barrier(world)
    torch.cuda.synchronize()
    e2e_start.record(stream)
    for _ in range(e2e_iters):
        rt.set_cell_words(pinned_offsets, pinned_words)
        rt.advance(seed=1000 + gen, counts=counts, config=cfg)
        e2e_steps += rt.stats().game_steps
        _ = rt.summary().best_fitness
        gen += 1
    e2e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e2e_start.elapsed_time(e2e_end), world)
    e2e_total = sum_over_ranks(float(e2e_steps), world)

    # ---- the plain FP32 form on the same workload, and the trunk form's agreement with it ----
    plain = None
    agree = None
    if args.form != "fp32" and not args.no_plain:
        if rank == 0 and trunk_form:
            agree = agreement_sample(rt, torch, counts, FORMS[args.form], args.tau, 3 * wl.secrets_per_cell)
        rt.set_form(0)
        for _ in range(1):
            rt.advance(seed=1000 + gen, counts=counts, config=cfg)
            gen += 1
        pagg, gen = time_generations(rt, torch, stream, world, local, args.steps, gen, counts, cfg)
        plain_value = sum_over_ranks(float(pagg["steps"]), world) / (pagg["ms"] * 1e-3)
        plain = {"value": plain_value, "unit": "game-steps/s", "ms_per_step": pagg["ms"] / args.steps,
                 "eval_kernel_ms": sum(pagg["kernel_ms"]) / len(pagg["kernel_ms"]),
                 "speedup_of_this_form": (total_steps / (ms * 1e-3)) / plain_value,
                 "note": "plain FP32 form, same workload and process, after this form's timed generations"}

    if rank != 0:
        rt.close()
        return
    race = None
    if world == 1 and not args.no_surrogate and args.workload == "full":
        rt.close()
        rt = None
        race = surrogate_vs_plain(nwg, wl, torch, args.surrogate_generations)
    pk = peaks()
    mean_steps = steps / args.steps
    mean_encoded = agg["encoded"] / args.steps
    kernel_mean_ms = sum(agg["kernel_ms"]) / len(agg["kernel_ms"])
    flops = algorithmic_flops(int(mean_steps), int(mean_encoded), wl.action_count)
    achieved_tflops = flops / (kernel_mean_ms * 1e-3) / 1e12
    fp32_peak = 148 * 128 * 2 * pk["sm_max_mhz"] * 1e6 / 1e12
    traffic_file = TRAFFIC_TCT if trunk_form else TRAFFIC
    traffic = None
    if traffic_file.exists() and (trunk_form or args.form == "fp32"):
        traffic = json.loads(traffic_file.read_text()).get("bytes_per_launch")
    if trunk_form or args.form in ("tc-bf16", "tc-fp16"):
        kernel = "EvalTctKernel" if trunk_form else "EvalTcKernel"
        roofline = {"kernel": kernel, "bound": "tensor", "achieved": achieved_tflops, "peak": pk["bf16_tflops"],
                    "unit": "TFLOP/s", "frac": achieved_tflops / pk["bf16_tflops"], "traffic": traffic,
                    "peak_source": f"dense bf16 burst ({pk['source']}); fp16 operands run at the same rate",
                    "frac_of_fp32_peak": achieved_tflops / fp32_peak}
    else:
        roofline = {"kernel": "EvalFp32Kernel", "bound": "fp32", "achieved": achieved_tflops, "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": achieved_tflops / fp32_peak, "traffic": traffic,
                    "peak_source": f"148 SMs x 128 FFMA/clk x 2 x {pk['sm_max_mhz']:.0f} MHz "
                                   f"(sm_max_mhz {pk['source']})",
                    "frac_of_bf16_tensor_peak": achieved_tflops / pk["bf16_tflops"]}
    roofline.update({"kernel_ms_per_launch": kernel_mean_ms, "algorithmic_flop_per_launch": flops,
                     "game_steps_per_launch": mean_steps})
    value = total_steps / (ms * 1e-3)
    line = {
        "metric": "game-steps/s",
        "value": value,
        "unit": "game-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": DTYPES[args.form],
        "data": "synthetic",
        "impl": "ours",
        "generations_per_s": args.steps / (ms * 1e-3),
        "config": {"workload": wl.name, "population": wl.population, "grid": f"{wl.population // wl.columns}x"
                   f"{wl.columns}", "action_count": wl.action_count, "secrets_per_cell": wl.secrets_per_cell,
                   "secret_subset": wl.secret_subset, "episodes_per_secret": 3, "selection_radius": wl.radius,
                   "mutation_probability": wl.mutation_probability, "mutation_sigma": wl.mutation_sigma,
                   "form": FORM_NAMES[args.form], "margin_tau": args.tau if trunk_form else None,
                   "parallelism": f"{world} independent populations (one per GPU)",
                   "l2": "inputs larger than L2 (genome slab "
                         f"{wl.population * nwg.capi.genome_stride_bytes(wl.action_count) / 1e9:.2f} GB)"},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_total / (e2e_ms * 1e-3), "unit": "game-steps/s",
                "h2d_bytes_per_step": int(offsets.nbytes + words.nbytes + 120),
                "d2h_bytes_per_step": 4 + 48 + 24},
        "gpu_launches": (KERNELS_PER_GENERATION + EXTRA_KERNELS[args.form]) * args.steps,
        "rescoring": {"chunks_per_step": agg["rescored"] / max(steps, 1),
                      "full_rescore_fraction": agg["full"] / max(steps, 1),
                      "candidate_chunks_per_step": agg["candidates"] / max(steps, 1),
                      "fallback_fraction": agg["fallbacks"] / max(steps, 1)},
        "plain_fp32": plain,
        "agreement_with_plain": agree,
        "surrogate_vs_plain": race,
        "clocks": agg["clocks"],
    }
    print(json.dumps(line), flush=True)
    if rt is not None:
        rt.close()


def run_growth(args) -> None:
    """Batching form with uneven shards: 16,384 individuals on a 128x128 grid, per-cell secret lists of
    floor(exp(U[ln 32, ln 1024])) words drawn from the first 1,024 catalog words, and the action space widened
    from 1,024 to 4,739 words in steps of 512 (the last step 131) over 50 generations. Every generation that does
    not widen runs as one CUDA graph with launch shapes tuned per width (nwg_advance_graphed); a widening
    generation breeds into the wider slab and injects the new rows directly. As in the reference, the generation
    byte budget is fixed at creation (16,384 genomes at 1,024 words), so each widening keeps the whole grid rows
    that still fit; the surviving cells keep their secret lists. Timed on the host with the device synchronised
    around each generation; game steps are counted on the device."""
    import torch

    rank, world, local = dist_setup(args.gpus)
    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    W, capi = nwg.workload, nwg.capi
    population, columns, start, final, step, generations = 16384, 128, 1024, 4739, 512, 50
    widths = list(range(start + step, final, step)) + [final]
    widen_at = {round((i + 1) * generations / (len(widths) + 1)): w for i, w in enumerate(widths)}
    # words past the starting width are injected later, so each needs a hint-grid group (a monochrome word, for
    # one, has none and the reference rejects its injection): draw replacements for those that lack one
    pool = W.synthetic_words(2 * final, 0)
    usable = capi.hint_groups_available(pool)
    tail = [w for w, ok in zip(pool[start:], usable[start:]) if ok][:final - start]
    catalog = np.concatenate([pool[:start], np.array(tail, np.uint8)])
    assert len(catalog) == final
    capi.upload_catalog(catalog)
    subset = W.secret_subset(start, start, 0)
    offsets, words = W.loguniform_cell_lists(population, 32, 1024, subset, rank)
    rt = nwg.Runtime(start, population, columns, stream=torch.cuda.current_stream().cuda_stream)
    rt.set_cell_words(offsets, words)
    rt.set_form(FORMS[args.form])
    if args.form.startswith("tc-trunk"):
        rt.set_margin_guard(args.tau)
    rt.bootstrap(population, seed=rank)
    cfg = capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    width = start
    per_width = {}
    total_steps, total_s = 0, 0.0
    with ClockSampler(local) as clocks:
        for g in range(generations):
            counts = capi.word_counts(training=start, action_space=width)
            pending = None
            if g in widen_at:
                pending = capi.PendingInjection(True, width, widen_at[g] - width)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rt.advance_graphed(seed=9000 + g, counts=counts, config=cfg, pending=pending)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            steps = rt.stats().game_steps
            total_steps += steps
            total_s += dt
            row = per_width.setdefault(width, {"generations": 0, "game_steps": 0, "seconds": 0.0})
            row["generations"] += 1
            row["game_steps"] += steps
            row["seconds"] += dt
            if pending is not None:
                width = widen_at[g]
                n = len(rt.current_generation()["slots"])
                rt.set_cell_words(offsets[:n + 1], words[:offsets[n]])
    tuning = {}
    for w in per_width:
        t = rt.launch_tuning(width=w)
        tuning[w] = {"decided": bool(t.decided), "eval_ctas": t.eval_ctas, "breed_warps": t.breed_warps,
                     "eval_ms": [round(x, 3) for x in t.eval_ms], "breed_ms": [round(x, 3) for x in t.breed_ms]}
    gi = rt.graph_info()
    value = sum_over_ranks(float(total_steps), world) / max_over_ranks(total_s, world)
    if rank == 0:
        print(json.dumps({
            "metric": "game-steps/s", "value": value, "unit": "game-steps/s", "n_gpus": world, "steps": generations,
            "warmup": 0, "ms_per_step": 1e3 * total_s / generations, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES[args.form], "data": "synthetic", "impl": "ours",
            "generations_per_s": generations / total_s,
            "config": {"workload": "p16384_grid128_a1024to4739_loguniform32to1024", "population": population,
                       "grid": "128x128", "action_width": f"{start} -> {final} in steps of {step}",
                       "widen_at_generation": widen_at, "secrets_per_cell": "floor(exp(U[ln 32, ln 1024]))",
                       "secret_words": f"the first {start} catalog words", "form": FORM_NAMES[args.form],
                       "margin_tau": args.tau, "timing": "host clock around each generation, device synchronised",
                       "final_population": len(rt.current_generation()["slots"]), "final_width": width},
            "per_width": {w: {**r, "game_steps_per_s": r["game_steps"] / r["seconds"]} for w, r in per_width.items()},
            "launch_tuning": tuning,
            "graphs": {"launches": gi.launches, "instantiations": gi.instantiations, "updates": gi.updates},
            "clocks": clocks.summary(),
        }), flush=True)
    rt.close()


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import pyoracle as O

    nwg_workload = importlib.import_module("neuroevolutionary-wordle_b200.workload")
    if args.workload == "growth":
        print(json.dumps({"impl": "reference", "unavailable": "the reference's CPU path has no widening run to time; "
                          "its arm is measured on the full workload"}))
        return
    wl = {"full": nwg_workload.FULL, "medium": nwg_workload.MEDIUM, "small": nwg_workload.SMALL}[args.workload]
    if O.ref_host() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_host.so was not built"}))
        return
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    threads = os.cpu_count() or 1
    sample = max(2, threads)
    rng = np.random.default_rng(0)
    halfs = 150528 + 38 * wl.action_count
    stds = [np.sqrt(2.0 / 145)] * (128 * 145) + [0.0] * 128 + [np.sqrt(2.0 / 128)] * (64 * 128) + [0.0] * 64 + \
        [np.sqrt(2.0 / 321)] * (256 * 321) + [0.0] * 256 + [np.sqrt(2.0 / 256)] * (128 * 256) + [0.0] * 128 + \
        [np.sqrt(2.0 / 128)] * (64 * 128) + [0.0] * 64 + [0.05] * (38 * wl.action_count)
    stds = np.array(stds, np.float32)
    assert len(stds) == halfs
    genomes = (rng.standard_normal((sample, halfs)).astype(np.float32) * stds).astype(np.float16).view(np.uint16)
    times = []
    steps_total = 0
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cells = ((np.arange(sample) + it * sample) % wl.population).astype(np.uint32)
        raw, steps, status = O.ref_host_evaluate(genomes, wl.action_count, catalog, offsets, words, cells, threads)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
            steps_total += int(steps.sum())
    total_s = sum(times)
    value = steps_total / total_s
    print(json.dumps({
        "metric": "game-steps/s", "value": value, "unit": "game-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (fp16-stored genomes)", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": wl.name, "population": wl.population, "action_count": wl.action_count,
                   "secrets_per_cell": wl.secrets_per_cell, "form": "reference CPU path",
                   "sample_per_step": f"evaluation of {sample} individuals"},
        "cpu_baseline": {"value": value, "unit": "game-steps/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} individuals per step, {steps_total} game steps timed"},
        "e2e": {"value": value, "unit": "game-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["full", "medium", "small", "growth"], default="full",
                    help="growth: the batching form (16,384 individuals, uneven shards, widening action space)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", choices=sorted(FORMS), default="tc-trunk-fp16")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison and the agreement sample")
    ap.add_argument("--tau", type=float, default=1e-3, help="margin guard of the tensor-core trunk forms (1e-3 x the score scale)")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate-vs-plain race")
    ap.add_argument("--surrogate-generations", type=int, default=50)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "growth":
        run_growth(args)
    else:
        run_ours(args)
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
