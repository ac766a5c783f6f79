"""Benchmark: one GA generation (evaluate, select, breed, mutate) per step on the B200.

Workload: population 4,096 on a 64x64 toroidal grid, 4,739 synthetic catalog words all active, 256
secrets per cell drawn from a 2,315-word secret subset (3 episodes per secret), radius-1 rank selection,
reference crossover temperatures, mutation p = 0.05, sigma = 0.02. Genomes are the reference's FP16
layout (bootstrap He-normal weights, N(0, 0.05) tails).

The headline form (default --form tc-fp16) gives the reference's results bit for bit: encoder, trunk and policy
are the reference's FP32 chains, 16-bit tensor-core scores only screen the actions, and every guess is the exact
FP32 argmax (the chunks a certified error bound cannot rule out are re-scored in FP32). Its line carries the
device-resident value, the same metric end to end through the public API with host buffers ("e2e"), the
evaluation kernel's roofline, and the reference's CPU path timed on the generation just measured
("cpu_baseline"). "other_forms" times the plain FP32 form (no tensor cores at all) and the 16-bit tensor-core
trunk forms (FP16 and BF16 operands, top-2 margin guard with exact FP32 fallback: narrower than the reference,
reported with their guess agreement against the plain form, "agreement_with_plain"). "reference_gpu" times the
reference's own CUDA evaluation (compiled for sm_100a from its sources) on a 256-individual slice of the workload
on the same GPU, beside this library's forms on the same slice.

On the full workload at N=1 the line also carries "batching_form", the widening run of the batching
configuration (16,384 individuals on 128x128, uneven per-cell lists, the action space widened from 1,024 to 4,739
words over 50 generations, graphed generations with tuned launch shapes, BF16 trunk form; --no-growth skips it),
and "surrogate" (--no-surrogate skips it): the learned network's pick against a random pick from the same broods
(95% interval over 24 generations) and the race against the plain form at the 0.6 audit floor, on the benchmark
workload and on a 256-word workload where the plain form learns and fitness ranks are reliable.

--gpus N (N > 1) starts N ranks on this node (or runs under torch.distributed.run) and splits the one population
into N row bands, one per GPU: evaluation per band, fitness all-gather, halo genome exchange with the neighbour
bands, breeding per band (strong scaling: the total work is the same as at N = 1).

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
TRAFFIC_FILES = {"fp32": ROOT / "profiles" / "eval_fp32_traffic.json",
                 "tc-fp16": ROOT / "profiles" / "eval_tc_traffic.json",
                 "tc-trunk-fp16": ROOT / "profiles" / "eval_tct_traffic.json"}
KERNELS_PER_GENERATION = 7  # prepare, evaluate, finalize, summarize, select, plan slots, breed
FORMS = {"fp32": 0, "tc-bf16": 1, "tc-fp16": 2, "tc-trunk-bf16": 3, "tc-trunk-fp16": 4}
FORM_NAMES = {"fp32": "plain fp32", "tc-bf16": "tensor-core bf16 scoring, exact fp32 re-scoring",
              "tc-fp16": "tensor-core fp16 scoring, exact fp32 re-scoring",
              "tc-trunk-bf16": "tensor-core bf16 encoder+trunk+scoring, margin guard tau with exact fp32 fallback",
              "tc-trunk-fp16": "tensor-core fp16 encoder+trunk+scoring, margin guard tau with exact fp32 fallback"}
EXTRA_KERNELS = {"fp32": 0, "tc-bf16": 1, "tc-fp16": 1, "tc-trunk-bf16": 2, "tc-trunk-fp16": 2}
# What each form's results are, against the reference's FP32 arithmetic.
PRECISION = {
    "fp32": "reference: every policy value, score and guess is the reference's FP32 chain, bit for bit",
    "tc-bf16": "reference: FP32 policy chains bit for bit; 16-bit tensor-core scores only screen actions and every "
               "guess is the exact FP32 argmax (certified error bound), so guesses, turns, scores and fitness are "
               "the reference's bit for bit",
    "tc-fp16": "reference: FP32 policy chains bit for bit; 16-bit tensor-core scores only screen actions and every "
               "guess is the exact FP32 argmax (certified error bound), so guesses, turns, scores and fitness are "
               "the reference's bit for bit",
    "tc-trunk-bf16": "narrower: 16-bit tensor-core policy; steps under the margin guard re-run in exact FP32",
    "tc-trunk-fp16": "narrower: 16-bit tensor-core policy; steps under the margin guard re-run in exact FP32",
}
DTYPES = {"fp32": "fp32 (fp16-stored genomes)",
          "tc-bf16": "fp32 (exact): fp32 trunk and decisions, bf16 tensor-core scores screen the actions",
          "tc-fp16": "fp32 (exact): fp32 trunk and decisions, fp16 tensor-core scores screen the actions",
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


def _surrogate_setup(nwg, wl):
    """Training and held-out per-cell secret lists (two seeded draws from the same secret subset), counts, config."""
    capi, W = nwg.capi, nwg.workload
    subset = W.secret_subset(wl.action_count, wl.secret_subset, wl.seed)
    train = wl.cell_lists()
    held = W.fixed_cell_lists(wl.population, wl.secrets_per_cell, subset, wl.seed + 101)
    counts = capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    return subset, train, held, counts, cfg


def _population(nwg, wl, form, train):
    rt = nwg.Runtime(wl.action_count, wl.population, wl.columns)
    rt.set_form(form)
    if form >= 3:
        rt.set_margin_guard(1e-3)
    rt.bootstrap(wl.population, seed=7)
    rt.set_cell_words(*train)
    return rt


def _heldout_rate(rt, counts, train, held):
    """Mean solve rate on the held-out secrets; the training fitness is evaluated again afterwards (deterministic),
    for the next selection."""
    rt.set_cell_words(*held)
    rt.evaluate(counts)
    rate = rt.solve_rates()[1]
    rt.set_cell_words(*train)
    rt.evaluate(counts)
    return rate


def _ranks(v):
    return np.argsort(np.argsort(v, kind="stable"), kind="stable").astype(np.float64)


def _test_retest(rt, counts, train, held):
    """Spearman of one population's fitness measured on the training and on the held-out secrets: how reliable one
    measured fitness is. No predictor's audit Spearman against measured fitness can exceed about its square root."""
    rt.set_cell_words(*train)
    rt.evaluate(counts)
    f_train = rt.current_generation()["fitness"].copy()
    rt.set_cell_words(*held)
    rt.evaluate(counts)
    f_held = rt.current_generation()["fitness"].copy()
    rt.set_cell_words(*train)
    rt.evaluate(counts)
    return float(np.corrcoef(_ranks(f_train), _ranks(f_held))[0, 1])


def _mean_ci95(values):
    """Mean and two-sided 95% t-interval of per-generation values."""
    v = np.asarray(values, np.float64)
    n = len(v)
    if n < 2:
        return {"mean": float(v.mean()) if n else None, "ci95": None, "n": n}
    try:
        from scipy.stats import t as student_t

        q = float(student_t.ppf(0.975, n - 1))
    except ImportError:  # the normal quantile, slightly narrower
        q = 1.96
    half = q * float(v.std(ddof=1)) / np.sqrt(n)
    return {"mean": float(v.mean()), "ci95": [float(v.mean() - half), float(v.mean() + half)], "n": n}


def surrogate_ablation(nwg, wl, torch, generations: int = 24) -> dict:
    """The network's pick against a random pick from the same broods. Every cell breeds 4 candidates; every candidate
    is played (screening off), so each generation measures, on the same children, the mean training fitness of the
    child the network scores best in each cell, of candidate 0 (the candidates are exchangeable draws, so candidate
    0 is a random pick, and it is exactly the plain step's child) and of the best-measured child (an upper bound no
    predictor can beat). The ratio and the difference model - random per generation over `generations` generations
    after the network's first training, with 95% intervals: a difference interval above 0 means the network picks
    fitter children than chance."""
    capi = nwg.capi
    subset, train, held, counts, cfg = _surrogate_setup(nwg, wl)
    rt = _population(nwg, wl, 4, train)
    retest = _test_retest(rt, counts, train, held)
    sc = capi.SurrogateConfig(seed=3, spearman_floor=2.0, train_steps=32)  # a floor above 1: never screens
    sur = capi.Surrogate(rt, wl.catalog(), sc, secret_pool=subset)
    ratios, diffs, best, spearman, g = [], [], [], [], 0
    while len(ratios) < generations and g < generations + 8:
        st = sur.advance(7000 + g, counts, cfg)
        g += 1
        if st.mean_fitness_model_pick != st.mean_fitness_model_pick:  # untrained yet
            continue
        ratios.append(st.mean_fitness_model_pick / st.mean_fitness_first_candidate)
        diffs.append(st.mean_fitness_model_pick - st.mean_fitness_first_candidate)
        best.append(st.mean_fitness_best_candidate / st.mean_fitness_first_candidate)
        if st.spearman == st.spearman:
            spearman.append(float(st.spearman))
    sur.close()
    rt.close()
    r, d = _mean_ci95(ratios), _mean_ci95(diffs)
    return {"workload": wl.name, "model_pick_over_random_pick": r, "model_pick_minus_random_pick": d,
            "best_measured_over_random_pick": _mean_ci95(best),
            "audit_spearman_mean": float(np.mean(spearman)) if spearman else None,
            "fitness_test_retest_spearman": retest,
            "network_beats_random": bool(d["ci95"] is not None and d["ci95"][0] > 0.0),
            "per_generation": [round(x, 5) for x in ratios]}


def surrogate_race(nwg, wl, torch, generations: int = 50, floor: float = 0.6) -> dict:
    """Time to equal held-out fitness: the plain FP32 form against the surrogate method at the given audit floor.

    The plain form evolves `generations` generations (prepare + assemble, device-synced wall time); its population's
    held-out mean solve rate (the same cells, a second seeded secret draw, untimed) is the target. The surrogate
    method (4 candidates per cell, network screening while the audit Spearman is at least `floor`, full evaluation of
    every candidate otherwise) evolves from the same generation 0 for at most `generations` generations. A crossing
    counts as the network's only if at least one screened step came before it; otherwise the line says that the
    target was reached by full-evaluation steps (best-of-4 broods), which measures brood size, not the network."""
    capi = nwg.capi
    subset, train, held, counts, cfg = _surrogate_setup(nwg, wl)
    rt = _population(nwg, wl, 0, train)
    retest = _test_retest(rt, counts, train, held)
    start = _heldout_rate(rt, counts, train, held)
    plain_s, plain_trace = 0.0, []
    for g in range(generations):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rt.prepare(5000 + g, counts, config=cfg)
        rt.assemble()
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
        if (g + 1) % 10 == 0:
            plain_trace.append([g + 1, round(_heldout_rate(rt, counts, train, held), 6)])
    target = plain_trace[-1][1] if plain_trace and plain_trace[-1][0] == generations \
        else _heldout_rate(rt, counts, train, held)
    rt.close()

    rt = _population(nwg, wl, 4 if wl.action_count > 128 else 0, train)
    sc = capi.SurrogateConfig(seed=1, spearman_floor=floor, train_steps=32)
    sur = capi.Surrogate(rt, wl.catalog(), sc, secret_pool=subset)
    sur_s, reached, screened, rhos, trace = 0.0, None, 0, [], []
    for g in range(generations):
        st = sur.advance(9000 + g, counts, cfg)
        sur_s += st.ms_total * 1e-3
        screened += int(st.screened)
        if st.spearman == st.spearman:
            rhos.append(float(st.spearman))
        rate = _heldout_rate(rt, counts, train, held)
        trace.append([int(st.generation), round(rate, 6), bool(st.screened),
                      None if st.spearman != st.spearman else round(float(st.spearman), 3)])
        if reached is None and rate >= target:
            reached = {"generation": int(st.generation), "seconds": sur_s, "screened_steps_before": screened}
    sur.close()
    rt.close()
    by_network = bool(reached is not None and reached["screened_steps_before"] > 0)
    return {
        "workload": wl.name, "audit_floor": floor,
        "plain": {"generations": generations, "seconds": plain_s, "heldout_solve_rate_start": start,
                  "heldout_solve_rate_end": target, "trace": plain_trace},
        "surrogate": {"generations": generations, "seconds": sur_s, "screened_steps": screened,
                      "audit_spearman_max": max(rhos) if rhos else None,
                      "audit_spearman_mean": float(np.mean(rhos)) if rhos else None,
                      "crossing": reached, "trace": trace},
        "crossing_by_screened_steps": by_network,
        "time_ratio": (reached["seconds"] / plain_s) if by_network else None,
        "fitness_test_retest_spearman": retest,
    }


def surrogate_study(nwg, torch, race_generations: int = 50, ablation_generations: int = 24) -> dict:
    """The learned surrogate measured two ways, on the benchmark grid (4,739 words) and on a workload where the plain
    form learns within 50 generations and one measured fitness is reliable enough to rank (256 words, 256 secrets per
    cell from all 256): the ablation (network pick against a random pick from the same broods, 95% interval) and
    the race at the 0.6 audit floor. The audit Spearman of any predictor against measured fitness is capped near the
    square root of the fitness test-retest Spearman, so a workload whose test-retest is below 0.36 cannot screen at
    a 0.6 floor; the line says so rather than lowering the floor."""
    W = nwg.workload
    learnable = W.Workload("p4096_a256_s256", 4096, 64, 256, 256, 256)
    out = {"method": "4 candidates per cell; MLP 8192-512-128-1 on 128 probe-state descriptors, 32 Adam steps per "
                     "generation; the best-scored candidate of each cell played plus a 5% audit sample while the "
                     "audit Spearman is at least the floor, every candidate played otherwise"}
    for wl in (learnable, W.FULL):
        nwg.capi.upload_catalog(wl.catalog())
        entry = {"ablation": surrogate_ablation(nwg, wl, torch, ablation_generations)}
        retest = entry["ablation"]["fitness_test_retest_spearman"]
        entry["audit_ceiling"] = float(np.sqrt(max(retest, 0.0)))
        if wl is learnable or entry["audit_ceiling"] >= 0.6:
            entry["race"] = surrogate_race(nwg, wl, torch, race_generations)
        else:
            entry["race"] = ("not run: fitness test-retest Spearman %.3f caps the audit Spearman near %.2f, below "
                             "the 0.6 floor, so no step can screen" % (retest, entry["audit_ceiling"]))
        out[wl.name] = entry
    nwg.capi.upload_catalog(W.FULL.catalog())
    notes = []
    for name in (learnable.name, W.FULL.name):
        ab, race = out[name]["ablation"], out[name]["race"]
        ci = ab["model_pick_over_random_pick"]["ci95"]
        notes.append("%s: network pick / random pick %.4f (95%% %s)%s" % (
            name, ab["model_pick_over_random_pick"]["mean"], "n/a" if ci is None else "%.4f-%.4f" % tuple(ci),
            "" if ab["network_beats_random"] else ", not above chance"))
        if isinstance(race, dict) and not race["crossing_by_screened_steps"]:
            notes.append("%s: no screened step before the crossing at the %.1f floor (audit Spearman max %s), so "
                         "the race measures best-of-4 broods, not the network" % (
                             name, race["audit_floor"], race["surrogate"]["audit_spearman_max"]))
    out["conclusion"] = "; ".join(notes)
    return out


def kernel_launches(form: str) -> int:
    return KERNELS_PER_GENERATION + EXTRA_KERNELS[form]


def roofline(form: str, steps: float, encoded: float, action_count: int, kernel_ms: float, pk: dict,
             fp32_peak: float, traffic) -> dict:
    """The evaluation kernel against its bound. The per-step work is 2 * (E_new + 123,136 + 64 A) FLOP (E_new =
    9,472 per newly encoded turn): the encoder and trunk share (2 * (9,472 per encoded turn + 123,136 per step))
    runs as FP32 FFMA chains in the plain and exact forms, the scoring share (2 * 64 A per step) on CUDA cores
    (plain) or on tensor cores (the other forms). The bound is the pipe whose share takes longest at its measured
    peak."""
    flops = algorithmic_flops(int(steps), int(encoded), action_count)
    trunk = 2.0 * (9472.0 * encoded + 123136.0 * steps)
    return roofline_of(form, flops, trunk, steps, kernel_ms, pk, fp32_peak, traffic)


def roofline_of(form: str, flops: float, trunk: float, steps: float, kernel_ms: float, pk: dict, fp32_peak: float,
                traffic) -> dict:
    """roofline() from the work itself: `flops` in all, `trunk` of it on the FP32 pipe in the plain and exact forms
    (a run over several action widths sums its generations' work)."""
    scoring = flops - trunk
    t = kernel_ms * 1e-3
    kernel = {"fp32": "EvalFp32Kernel", "tc-bf16": "EvalTcKernel<bf16>", "tc-fp16": "EvalTcKernel<fp16>",
              "tc-trunk-bf16": "EvalTctKernel<bf16>", "tc-trunk-fp16": "EvalTctKernel<fp16>"}[form]
    common = {"kernel": kernel, "kernel_ms_per_launch": kernel_ms, "algorithmic_flop_per_launch": flops,
              "game_steps_per_launch": steps, "traffic": traffic,
              "fp32_peak_tflops": fp32_peak, "fp32_peak_source": pk["fp32_source"],
              "tensor_peak_tflops": pk["bf16_tflops"], "tensor_peak_source": f"dense bf16 burst ({pk['source']})"}
    if form == "fp32":
        achieved = flops / t / 1e12
        return {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, **common}
    if form in ("tc-bf16", "tc-fp16"):
        # FP32 chains for encoder and trunk; tensor-core scores with exact FP32 re-scores of the candidate chunks
        achieved = trunk / t / 1e12
        return {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "fp32_pipe_flop_per_launch": trunk,
                "tensor_flop_per_launch": scoring,
                "min_ms_at_peaks": 1e3 * (trunk / (fp32_peak * 1e12) + scoring / (pk["bf16_tflops"] * 1e12)),
                **common}
    achieved = flops / t / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": pk["bf16_tflops"], "unit": "TFLOP/s",
            "frac": achieved / pk["bf16_tflops"], "fp16 operands": "run at the bf16 rate", **common}


def form_line(rt, torch, stream, world, local, form, tau, steps, gen, counts, cfg, sample_clocks=False):
    """Times `steps` generations of `form` after one untimed generation at that form."""
    rt.set_form(FORMS[form])
    if form.startswith("tc-trunk"):
        rt.set_margin_guard(tau)
    rt.advance(seed=1000 + gen, counts=counts, config=cfg)
    gen += 1
    agg, gen = time_generations(rt, torch, stream, world, local, steps, gen, counts, cfg, sample_clocks)
    return agg, gen


def e2e_line(rt, torch, stream, world, offsets, words, counts, cfg, gen, iterations):
    """The metric through the public API with host buffers: every step uploads its cell lists from pinned host
    memory (nwg_set_cell_words), advances one generation and reads the summary back."""
    pinned_offsets = torch.from_numpy(offsets).pin_memory().numpy()
    pinned_words = torch.from_numpy(words).pin_memory().numpy()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    steps = 0
    barrier(world)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(iterations):
        rt.set_cell_words(pinned_offsets, pinned_words)
        rt.advance(seed=1000 + gen, counts=counts, config=cfg)
        steps += rt.stats().game_steps
        _ = rt.summary().best_fitness
        gen += 1
    end.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(end), world)
    total = sum_over_ranks(float(steps), world)
    return {"value": total / (ms * 1e-3), "unit": "game-steps/s",
            "h2d_bytes_per_step": int(offsets.nbytes + words.nbytes + 120), "d2h_bytes_per_step": 4 + 48 + 24,
            "steps": iterations, "ms_per_step": ms / iterations}, gen


def cpu_model() -> str:
    try:
        for line in subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return "unknown"


def cpu_baseline_on(rt, catalog, offsets, words, action_count, label):
    """The reference's CPU path (oracle/_ref/libref_host.so, every host thread) on genomes of the runtime's current
    generation with their own cells."""
    threads = os.cpu_count() or 1
    sample = min(len(rt.current_generation()["slots"]), max(2, threads))
    gen = rt.current_generation()
    genomes = np.stack([rt.download_slot(int(gen["slots"][i])).view(np.uint16) for i in range(sample)])
    res = cpu_reference_rate(catalog, offsets, words, genomes, action_count, sample, threads)
    if res is None:
        return None
    rate, dt, steps = res
    return {"value": rate, "unit": "game-steps/s", "cores": threads, "cpu": cpu_model(), "kind": "reference",
            "sample": f"{label}: evaluation of {sample} individuals (generation {gen['generation_index']}) with "
                      f"their own cells, {steps} game steps in {dt:.1f} s on {threads} threads"}


def reference_gpu(nwg, torch, wl, catalog, population=256, columns=16, repeats=3):
    """The reference's own CUDA evaluation on this B200: oracle/_ref/libref_ckpt.so (slab_runtime.cu compiled for
    sm_100a) runs TryEvaluateCurrentGenerationFitnessOnDevice (slab_runtime.cu:1086; warp scorer above 128
    actions, slab_runtime.cu:452-549) through its own API on a bootstrapped slice of the workload: `population`
    individuals at the full action space, each playing the 3 x 256 episodes of a 256-word foundation shard. This
    library evaluates the same genomes (its bootstrap is the reference's, bit for bit) and the same shard with the
    plain form and the exact tensor-core-screened form; their fitness must equal the reference's."""
    import ctypes as C

    from oracle import pyoracle as O

    L = O.ref_ckpt()
    if L is None:
        return {"unavailable": "oracle/_ref/libref_ckpt.so was not built"}
    capi = nwg.capi
    counts = capi.word_counts(training=wl.secrets_per_cell, action_space=wl.action_count)
    stride = capi.genome_stride_bytes(wl.action_count)
    rc = capi.RuntimeConfig()
    rc.genotype_slab_byte_budget_bytes = 2 * population * stride
    rc.generation_byte_budget_bytes = population * stride
    rc.action_count, rc.population_size_ceiling, rc.grid_column_count = wl.action_count, population, columns
    ms = np.zeros(repeats, np.float64)
    ref_fit = np.zeros(population, np.float32)
    letters = np.ascontiguousarray(catalog, np.uint8)
    seed = 11
    if L.refckpt_time_evaluation(C.addressof(rc), letters.ctypes.data, len(letters), population, seed, 0,
                                 C.addressof(counts), repeats, ms.ctypes.data, ref_fit.ctypes.data) != 1:
        return {"unavailable": "the reference runtime failed on the slice"}
    nwg.capi.upload_catalog(catalog)
    rt = nwg.Runtime(wl.action_count, population, columns, stream=torch.cuda.current_stream().cuda_stream)
    rt.bootstrap(population, seed=seed)
    ours = {}
    for form in ("fp32", "tc-fp16"):
        rt.set_form(FORMS[form])
        rt.evaluate(counts)  # warm-up (and the tables of the tensor-core form)
        times = []
        for _ in range(repeats):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rt.evaluate(counts)
            times.append(1e3 * (time.perf_counter() - t0))
        st = rt.stats()
        fit = rt.current_generation()["fitness"]
        ours[form] = {"ms": statistics.median(times), "game_steps": int(st.game_steps),
                      "fitness_equals_reference": bool(np.array_equal(fit.view(np.uint32), ref_fit.view(np.uint32)))}
    rt.close()
    steps = ours["fp32"]["game_steps"]
    ref_ms = float(np.median(ms[1:])) if repeats > 1 else float(ms[0])
    return {"value": steps / (ref_ms * 1e-3), "unit": "game-steps/s", "ms_per_evaluation": ref_ms,
            "ms_all_calls": [round(float(x), 2) for x in ms],
            "slice": f"{population} individuals ({population // columns}x{columns}) x {wl.action_count} actions, "
                     f"foundation shard of {wl.secrets_per_cell} words (768 episodes each), {steps} game steps",
            "what": "the reference's TryEvaluateCurrentGenerationFitnessOnDevice (slab_runtime.cu:1086) compiled for "
                    "sm_100a from its sources, host clock around each call (each synchronises)",
            "ours_same_slice": {f: {"value": o["game_steps"] / (o["ms"] * 1e-3), "ms_per_evaluation": o["ms"],
                                    "fitness_equals_reference": o["fitness_equals_reference"],
                                    "speedup_over_reference_gpu": ref_ms / o["ms"]} for f, o in ours.items()}}


def run_bands(args, nwg, torch, wl, rank, world, local) -> None:
    """N > 1: one population split by grid rows, one band per rank (nwg_set_band): fitness all-gathered, halo genomes
    exchanged with the neighbour bands, every band breeding its own rows. Total work is fixed (strong scaling)."""
    bands = importlib.import_module("neuroevolutionary-wordle_b200.bands")
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    nwg.capi.upload_catalog(catalog)
    layout = bands.band_layout(wl.population // wl.columns, wl.columns, world, rank, wl.radius)
    band = bands.BandRuntime(layout, wl.action_count)
    band.rt.set_form(FORMS[args.form])
    if args.form.startswith("tc-trunk"):
        band.rt.set_margin_guard(args.tau)
    band.bootstrap(0)
    band.set_cell_words(offsets, words)
    counts = nwg.capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = nwg.capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    stream = torch.cuda.current_stream()
    gen = 0
    for _ in range(args.warmup):
        band.advance(1000 + gen, counts, cfg)
        gen += 1
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    steps = 0
    kernel_ms = []
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.__enter__()
    start.record(stream)
    for _ in range(args.steps):
        band.advance(1000 + gen, counts, cfg)
        st = band.rt.stats()
        steps += st.game_steps
        kernel_ms.append(st.eval_kernel_ms)
        gen += 1
    end.record(stream)
    torch.cuda.synchronize()
    clocks.__exit__(None, None, None)
    barrier(world)
    ms = max_over_ranks(start.elapsed_time(end), world)
    total = sum_over_ranks(float(steps), world)
    # end to end: host cell lists uploaded every step, the band summary read back
    pinned_offsets = torch.from_numpy(offsets).pin_memory().numpy()
    pinned_words = torch.from_numpy(words).pin_memory().numpy()
    iters = max(1, min(args.steps, 3))
    e_steps = 0
    barrier(world)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(iters):
        band.set_cell_words(pinned_offsets, pinned_words)
        band.advance(1000 + gen, counts, cfg)
        e_steps += band.rt.stats().game_steps
        _ = band.rt.summary().best_fitness
        gen += 1
    end.record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(start.elapsed_time(end), world)
    e_total = sum_over_ranks(float(e_steps), world)
    mean, var = band.fitness_moments()  # whole grid, FP64 (one all-reduce of three sums)
    band_bytes = (layout.cells + 1) * 4 + int(offsets[layout.first_cell + layout.cells] - offsets[layout.first_cell]) * 4
    if rank == 0:
        print(json.dumps({
            "metric": "game-steps/s", "value": total / (ms * 1e-3), "unit": "game-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": DTYPES[args.form], "data": "synthetic",
            "impl": "ours", "generations_per_s": args.steps / (ms * 1e-3),
            "config": {"workload": wl.name, "population": wl.population,
                       "grid": f"{wl.population // wl.columns}x{wl.columns}", "action_count": wl.action_count,
                       "secrets_per_cell": wl.secrets_per_cell, "form": FORM_NAMES[args.form],
                       "parallelism": f"row bands: {world} bands of {layout.rows} rows, halo {layout.halo} row(s); "
                                      "fitness all-gather + halo genome exchange (NCCL) per generation",
                       "l2": "inputs larger than L2"},
            "e2e": {"value": e_total / (e_ms * 1e-3), "unit": "game-steps/s", "h2d_bytes_per_step": band_bytes + 120,
                    "d2h_bytes_per_step": 76},
            "gpu_launches": (kernel_launches(args.form) + 3) * args.steps,
            "eval_kernel_ms_rank0": sum(kernel_ms) / len(kernel_ms),
            "last_evaluation_fp64": {"fitness_mean": mean, "fitness_variance": var},
            "clocks": clocks.summary(),
        }), flush=True)
    band.close()


def run_ours(args) -> None:
    import torch

    rank, world, local = dist_setup(args.gpus)
    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    wl = {"full": nwg.workload.FULL, "quarter": nwg.workload.QUARTER, "medium": nwg.workload.MEDIUM,
          "small": nwg.workload.SMALL}[args.workload]
    if world > 1:
        run_bands(args, nwg, torch, wl, rank, world, local)
        return
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    nwg.capi.upload_catalog(catalog)
    stream = torch.cuda.current_stream()
    pk = peaks()
    fp32_peak = nwg.capi.measure_fp32_peak(stream.cuda_stream)
    pk["fp32_source"] = "measured live by nwg_measure_fp32_peak (independent FFMA chains on every SM)"
    rt = nwg.Runtime(wl.action_count, wl.population, wl.columns, stream=stream.cuda_stream)
    rt.set_cell_words(offsets, words)
    rt.bootstrap(wl.population, seed=0)
    counts = nwg.capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = nwg.capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    form = args.form
    rt.set_form(FORMS[form])
    if form.startswith("tc-trunk"):
        rt.set_margin_guard(args.tau)
    gen = 0
    for _ in range(args.warmup):
        rt.advance(seed=1000 + gen, counts=counts, config=cfg)
        gen += 1

    # ---- the headline form, device-resident ----
    agg, gen = time_generations(rt, torch, stream, world, local, args.steps, gen, counts, cfg, sample_clocks=True)
    ms = agg["ms"]
    steps = agg["steps"]
    value = steps / (ms * 1e-3)
    traffic_file = TRAFFIC_FILES.get(form)
    traffic = json.loads(traffic_file.read_text()).get("bytes_per_launch") if traffic_file and traffic_file.exists() \
        else None
    kernel_mean_ms = sum(agg["kernel_ms"]) / len(agg["kernel_ms"])
    line_roofline = roofline(form, steps / args.steps, agg["encoded"] / args.steps, wl.action_count, kernel_mean_ms,
                             pk, fp32_peak, traffic)

    # ---- the headline form end to end through the public API ----
    e2e, gen = e2e_line(rt, torch, stream, world, offsets, words, counts, cfg, gen, max(1, min(args.steps, 3)))

    # ---- the CPU baseline on the generation just timed ----
    cpu = None if args.no_cpu_baseline else cpu_baseline_on(rt, catalog, offsets, words, wl.action_count,
                                                             "the timed run's latest generation")

    others = {}
    agreement = {}
    if not args.no_plain:
        for other in [f for f in ("fp32", "tc-trunk-fp16", "tc-trunk-bf16") if f != form]:
            oagg, gen = form_line(rt, torch, stream, world, local, other, args.tau, args.steps, gen, counts, cfg)
            o_kernel = sum(oagg["kernel_ms"]) / len(oagg["kernel_ms"])
            o_value = oagg["steps"] / (oagg["ms"] * 1e-3)
            entry = {"value": o_value, "unit": "game-steps/s", "ms_per_step": oagg["ms"] / args.steps,
                     "generations_per_s": args.steps / (oagg["ms"] * 1e-3), "dtype": DTYPES[other],
                     "form": FORM_NAMES[other],
                     "roofline": roofline(other, oagg["steps"] / args.steps, oagg["encoded"] / args.steps,
                                          wl.action_count, o_kernel, pk, fp32_peak,
                                          (json.loads(TRAFFIC_FILES[other].read_text()).get("bytes_per_launch")
                                           if other in TRAFFIC_FILES and TRAFFIC_FILES[other].exists() else None))}
            if other.startswith("tc-trunk"):
                entry["margin_tau"] = args.tau
                entry["rescoring"] = {"candidate_chunks_per_step": oagg["candidates"] / max(oagg["steps"], 1),
                                      "fallback_fraction": oagg["fallbacks"] / max(oagg["steps"], 1)}
                if other == "tc-trunk-fp16":
                    entry["e2e"], gen = e2e_line(rt, torch, stream, world, offsets, words, counts, cfg, gen,
                                                 max(1, min(args.steps, 3)))
            others[other] = entry
        plain_value = others["fp32"]["value"] if "fp32" in others else value
        for name, entry in others.items():
            entry["speedup_over_plain_fp32"] = entry["value"] / plain_value
        # guess agreement of the 16-bit trunk forms and of the headline with the plain form, whole population
        for f in [x for x in (form, "tc-trunk-fp16", "tc-trunk-bf16") if x != "fp32"]:
            agreement[f] = agreement_sample(rt, torch, counts, FORMS[f], args.tau, 3 * wl.secrets_per_cell)

    ref_gpu = None
    if not args.no_reference_gpu and args.workload == "full":
        ref_gpu = reference_gpu(nwg, torch, wl, catalog)
        nwg.capi.upload_catalog(catalog)
    if rt is not None:
        rt.close()
        rt = None
    batching = None
    if not args.no_growth and args.workload == "full":
        # config 3 names BF16 operands for the batching form
        batching = growth_run(nwg, torch, "tc-trunk-bf16", args.tau, 0, local, world, extras=True)
        for k in ("total_steps", "total_s"):
            batching.pop(k)
        nwg.capi.upload_catalog(catalog)
    race = None
    if not args.no_surrogate and args.workload == "full":
        race = surrogate_study(nwg, torch, args.surrogate_generations)
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
        "dtype": DTYPES[form],
        "precision": PRECISION[form],
        "data": "synthetic",
        "impl": "ours",
        "generations_per_s": args.steps / (ms * 1e-3),
        "config": {"workload": wl.name, "population": wl.population, "grid": f"{wl.population // wl.columns}x"
                   f"{wl.columns}", "action_count": wl.action_count, "secrets_per_cell": wl.secrets_per_cell,
                   "secret_subset": wl.secret_subset, "episodes_per_secret": 3, "selection_radius": wl.radius,
                   "mutation_probability": wl.mutation_probability, "mutation_sigma": wl.mutation_sigma,
                   "form": FORM_NAMES[form], "margin_tau": args.tau if form.startswith("tc-trunk") else None,
                   "parallelism": "one GPU, the whole population",
                   "l2": "inputs larger than L2 (genome slab "
                         f"{wl.population * nwg.capi.genome_stride_bytes(wl.action_count) / 1e9:.2f} GB)"},
        "roofline": line_roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": kernel_launches(form) * args.steps,
        "rescoring": {"chunks_per_step": agg["rescored"] / max(steps, 1),
                      "full_rescore_fraction": agg["full"] / max(steps, 1),
                      "candidate_chunks_per_step": agg["candidates"] / max(steps, 1),
                      "fallback_fraction": agg["fallbacks"] / max(steps, 1)},
        "other_forms": others or None,
        "agreement_with_plain": agreement or None,
        "reference_gpu": ref_gpu,
        "batching_form": batching,
        "surrogate": race,
        "clocks": agg["clocks"],
    }
    print(json.dumps(line), flush=True)
    if rt is not None:
        rt.close()


def growth_run(nwg, torch, form: str, tau: float, rank: int = 0, local: int = 0, world: int = 1,
               extras: bool = False, cpu: bool = False) -> dict:
    """Batching form with uneven shards (the widening run): 16,384 individuals on a 128x128 grid, per-cell secret
    lists of floor(exp(U[ln 32, ln 1024])) words drawn from the first 1,024 catalog words, and the action space
    widened from 1,024 to 4,739 words in steps of 512 (the last step 131) over 50 generations. Every generation that
    does not widen runs as one CUDA graph with launch shapes tuned per width (nwg_advance_graphed); a widening
    generation breeds into the wider slab and injects the new rows directly. As in the reference, the generation
    byte budget is fixed at creation (16,384 genomes at 1,024 words), so each widening keeps the whole grid rows
    that still fit; the surviving cells keep their secret lists. Timed on the host with the device synchronised
    around each generation; game steps are counted on the device. Returns this rank's totals and the line fields;
    with `extras`, also the evaluation kernel's roofline over the whole run, the end-to-end metric at the final
    width (host buffers) and, with `cpu`, the reference's CPU path on the final generation."""
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
    rt.set_form(FORMS[form])
    if form.startswith("tc-trunk"):
        rt.set_margin_guard(tau)
    rt.bootstrap(population, seed=rank)
    cfg = capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    width = start
    per_width = {}
    total_steps, total_s = 0, 0.0
    work = {"flops": 0.0, "trunk": 0.0, "kernel_ms": 0.0}
    cur_offsets, cur_words = offsets, words
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
            st = rt.stats()
            steps = st.game_steps
            total_steps += steps
            total_s += dt
            work["flops"] += algorithmic_flops(steps, st.encoded_turns, width)
            work["trunk"] += 2.0 * (9472.0 * st.encoded_turns + 123136.0 * steps)
            work["kernel_ms"] += st.eval_kernel_ms
            row = per_width.setdefault(width, {"generations": 0, "game_steps": 0, "seconds": 0.0})
            row["generations"] += 1
            row["game_steps"] += steps
            row["seconds"] += dt
            if pending is not None:
                width = widen_at[g]
                n = len(rt.current_generation()["slots"])
                cur_offsets, cur_words = offsets[:n + 1], words[:offsets[n]]
                rt.set_cell_words(cur_offsets, cur_words)
    tuning = {}
    for w in per_width:
        t = rt.launch_tuning(width=w)
        tuning[w] = {"decided": bool(t.decided), "eval_ctas": t.eval_ctas, "breed_warps": t.breed_warps,
                     "eval_ms": [round(x, 3) for x in t.eval_ms], "breed_ms": [round(x, 3) for x in t.breed_ms]}
    gi = rt.graph_info()
    final_population = len(rt.current_generation()["slots"])
    more = {}
    if extras:
        stream = torch.cuda.current_stream()
        pk = peaks()
        fp32_peak = nwg.capi.measure_fp32_peak(stream.cuda_stream)
        pk["fp32_source"] = "measured live by nwg_measure_fp32_peak (independent FFMA chains on every SM)"
        line_roofline = roofline_of(form, work["flops"], work["trunk"], total_steps, work["kernel_ms"], pk,
                                    fp32_peak, None)
        for k in ("algorithmic_flop_per_launch", "game_steps_per_launch", "fp32_pipe_flop_per_launch",
                  "tensor_flop_per_launch", "min_ms_at_peaks"):
            if k in line_roofline:
                line_roofline[k] /= generations
        line_roofline["kernel_ms_per_launch"] = work["kernel_ms"] / generations
        line_roofline["over"] = f"all {generations} generations (every width): work and kernel time summed, " \
                                "per-launch fields their means"
        counts = capi.word_counts(training=start, action_space=width)
        e2e, _ = e2e_line(rt, torch, stream, world, cur_offsets, cur_words, counts, cfg, 9000 + generations, 3)
        e2e["at"] = f"the final width ({width} words, {final_population} individuals), ungraphed advance"
        more = {"roofline": line_roofline, "e2e": e2e}
        if cpu:
            more["cpu_baseline"] = cpu_baseline_on(rt, catalog, cur_offsets, cur_words, width,
                                                   f"widening run at its final width ({width} words)")
    rt.close()
    return {**more,
        "total_steps": total_steps, "total_s": total_s, "generations": generations,
        "value": total_steps / total_s, "unit": "game-steps/s", "generations_per_s": generations / total_s,
        "ms_per_generation": 1e3 * total_s / generations, "dtype": DTYPES[form],
        "config": {"workload": "p16384_grid128_a1024to4739_loguniform32to1024", "population": population,
                   "grid": "128x128", "action_width": f"{start} -> {final} in steps of {step}",
                   "widen_at_generation": widen_at, "secrets_per_cell": "floor(exp(U[ln 32, ln 1024]))",
                   "secret_words": f"the first {start} catalog words", "form": FORM_NAMES[form],
                   "margin_tau": tau if form.startswith("tc-trunk") else None,
                   "timing": "host clock around each generation, device synchronised",
                   "final_population": final_population, "final_width": width},
        "per_width": {w: {**r, "game_steps_per_s": r["game_steps"] / r["seconds"]} for w, r in per_width.items()},
        "launch_tuning": tuning,
        "graphs": {"launches": gi.launches, "instantiations": gi.instantiations, "updates": gi.updates},
        "clocks": clocks.summary(),
    }


def run_growth(args) -> None:
    """The widening run alone (growth_run), one JSON line; every rank runs its own 16,384-individual grid."""
    import torch

    rank, world, local = dist_setup(args.gpus)
    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    r = growth_run(nwg, torch, args.form, args.tau, rank, local, world, extras=True,
                   cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    value = sum_over_ranks(float(r["total_steps"]), world) / max_over_ranks(r["total_s"], world)
    if rank == 0:
        print(json.dumps({
            "metric": "game-steps/s", "value": value, "unit": "game-steps/s", "n_gpus": world,
            "steps": r["generations"], "warmup": 0, "ms_per_step": r["ms_per_generation"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": r["dtype"], "data": "synthetic", "impl": "ours",
            "generations_per_s": r["generations_per_s"], "config": r["config"], "per_width": r["per_width"],
            "roofline": r.get("roofline"), "cpu_baseline": r.get("cpu_baseline"), "e2e": r.get("e2e"),
            "gpu_launches": kernel_launches(args.form) * r["generations"],
            "launch_tuning": r["launch_tuning"], "graphs": r["graphs"], "clocks": r["clocks"],
        }), flush=True)


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
    wl = {"full": nwg_workload.FULL, "quarter": nwg_workload.QUARTER, "medium": nwg_workload.MEDIUM,
          "small": nwg_workload.SMALL}[args.workload]
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
    generation = cpu_generation_small(O, wl, catalog, offsets, words, threads) if args.workload == "small" else None
    print(json.dumps({
        "metric": "game-steps/s", "value": value, "unit": "game-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (fp16-stored genomes)", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": wl.name, "population": wl.population, "action_count": wl.action_count,
                   "secrets_per_cell": wl.secrets_per_cell, "form": "reference CPU path",
                   "sample_per_step": f"evaluation of {sample} individuals"},
        "cpu_baseline": {"value": value, "unit": "game-steps/s", "cores": threads, "cpu": cpu_model(),
                         "kind": "reference",
                         "sample": f"{sample} individuals per step, {steps_total} game steps timed"},
        "e2e": {"value": value, "unit": "game-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_generation": generation,
    }), flush=True)


def cpu_generation_small(O, wl, catalog, offsets, words, threads: int) -> dict | None:
    """One whole generation of the 64-individual configuration on the host cores: the reference's CPU evaluation of
    every individual (libref_host, every host thread), then cellular rank selection and breeding of the 64 children
    by the oracle's single-thread restatement (the reference has no host selection or breeding). The Philox draws
    those two steps consume are recorded on the GPU by the generator itself beforehand (oracle/nwg_tape.cu) and are
    not part of the host time."""
    try:
        import torch
    except ImportError:
        return None
    if not torch.cuda.is_available():
        return None
    try:
        tl = O.tape_lib()
    except OSError:
        return None
    n, cols = wl.population, wl.columns
    rows = n // cols
    halfs = O.genome_halfs(wl.action_count)
    rng = np.random.default_rng(5)
    genomes = (rng.standard_normal((n, halfs)).astype(np.float32) * 0.05).astype(np.float16).view(np.uint16)
    seed, gen_index, radius, exponent = 77, 1, wl.radius, 0.5
    cfg = {"l1": 0.02, "l2": 0.01, "l3": 0.005, "p": wl.mutation_probability, "sigma": wl.mutation_sigma}
    draws = torch.zeros(6 * n, dtype=torch.int32, device="cuda")
    weights = torch.zeros(32, dtype=torch.float32, device="cuda")
    assert tl.tape_selection_draws(seed, gen_index, n, draws.data_ptr()) == 1
    assert tl.tape_pow_table(exponent, 32, weights.data_ptr()) == 1
    d = draws.cpu().numpy().view(np.uint32).reshape(n, 6)
    w = weights.cpu().numpy()
    O.set_fma_mode(True)
    t0 = time.perf_counter()
    raw_fit, steps, _ = O.ref_host_evaluate(genomes, wl.action_count, catalog, offsets, words,
                                            np.arange(n, dtype=np.uint32), threads)
    t1 = time.perf_counter()
    fitness = np.array([O.normalize_fitness(float(r), wl.secrets_per_cell) for r in raw_fit], np.float32)
    pairs = [O.select_parent_pair(fitness, np.ones(n, np.uint8), rows, cols, rows, c, radius, d[c], w)
             for c in range(n)]
    t2 = time.perf_counter()
    # each child's draws are recorded on the GPU just before its host breeding, which alone is timed
    length = 3 * halfs + 64
    raw = torch.zeros(length, dtype=torch.int32, device="cuda")
    uni = torch.zeros(length, dtype=torch.float32, device="cuda")
    nrm = torch.zeros(2 * length, dtype=torch.float32, device="cuda")
    breed_s = 0.0
    for c, (a, b) in enumerate(pairs):
        assert tl.tape_positions(seed, (c + gen_index * 4099) & 0xFFFFFFFF, length, raw.data_ptr(), uni.data_ptr(),
                                 nrm.data_ptr()) == 1
        tape = dict(raw=raw.cpu().numpy().view(np.uint32), uniform=uni.cpu().numpy(), normal_pair=nrm.cpu().numpy())
        tb = time.perf_counter()
        child = O.breed_and_mutate(genomes[a], genomes[b], wl.action_count, tape, cfg)
        breed_s += time.perf_counter() - tb
        if child is None:
            return None
    total = (t2 - t0) + breed_s
    t3 = t2 + breed_s
    return {"generations_per_s": 1.0 / total, "seconds": total, "evaluate_s": t1 - t0, "select_s": t2 - t1,
            "breed_s": t3 - t2, "game_steps": int(steps.sum()), "cores_evaluate": threads, "cores_select_breed": 1,
            "what": f"{n} individuals on {rows}x{cols}, {wl.action_count} words, {wl.secrets_per_cell} secrets per "
                    "cell: evaluation by the reference's host code, selection and breeding by the oracle's "
                    "restatement from Philox draws recorded on the GPU beforehand (not timed)"}


def launch_ranks(args) -> None:
    """`--gpus N` outside a launcher: start N ranks (one process per GPU) under torch.distributed.run on this node
    and exit with their status. Under a launcher whose world size differs from N, refuse."""
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if world == args.gpus or (world == 0 and args.gpus == 1):
        return
    if world != 0 or args.gpus < 1:
        print(json.dumps({"error": f"--gpus {args.gpus} but the launcher started {world} rank(s)"}), file=sys.stderr)
        sys.exit(2)
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
    sys.exit(subprocess.call(cmd))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["full", "quarter", "medium", "small", "growth"], default="full",
                    help="growth: the batching form (16,384 individuals, uneven shards, widening action space)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", choices=sorted(FORMS), default="tc-fp16",
                    help="headline form (default: FP32 trunk and decisions, tensor-core screening; results "
                         "bit-identical to the reference's)")
    ap.add_argument("--no-plain", action="store_true", help="skip the other forms and the agreement samples")
    ap.add_argument("--tau", type=float, default=1e-3, help="margin guard of the tensor-core trunk forms (1e-3 x the score scale)")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate ablation and race")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA evaluation on a slice of the workload")
    ap.add_argument("--surrogate-generations", type=int, default=50, help="generations of the surrogate race")
    ap.add_argument("--no-growth", action="store_true",
                    help="skip the widening run (16,384 individuals, 1,024 -> 4,739 words) in the full line")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    launch_ranks(args)
    if args.workload == "growth":
        run_growth(args)
    else:
        run_ours(args)
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
