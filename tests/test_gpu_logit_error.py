"""Logits and per-individual fitness of the precision form against an FP64 host oracle.

1,024 individuals (a 32x32 grid) at 4,739 actions play the first 256 of their games (86 secrets per cell, three
episodes each) in the plain FP32 form and in the FP16 tensor-core trunk form (margin guard 1e-3), with traces.
On the host, in FP64:
  * every traced decision state is rebuilt (secret e/3, prefill words e/3+1, e/3+2 or e/3+3, e/3+4 of the cell's
    list, then the traced choices; Wordle feedback by the reference's rules) and its policy vector recomputed
    (encoder 145 -> 128 ReLU -> 64 per turn, virgin flag and five turn slots, trunk 321 -> 256 ReLU -> 128 ReLU
    -> 64) from the genome's FP16 weights;
  * logits are that policy against each action's embedding (26 letter counts, -1 for an absent letter, then the
    38 FP16 tail values), and the tensor-core form's logits are its traced policy rounded to FP16 against the
    same embeddings (the products the tensor cores form; their FP32 accumulation adds at most 64 ulps);
  * every individual's 256 games are replayed with FP64 argmax guesses (guessed words masked, ties to the lower
    index), giving its FP64 raw score (10 + 6 - turns per won game).
The plain form's policies must match the FP64 recomputation to FP32 rounding, which pins the host replay; the
tensor-core form's policy and logit errors and both forms' per-individual fitness deltas are bounded and
printed. Reference layout: model/policy_model/policy_model.hpp, shared_encoder.hpp, dense_trunk.hpp,
output_embedding.hpp, wordle/feedback.hpp, evaluation_ops.cuh:171-242.
"""
import json

import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G

pytestmark = pytest.mark.gpu

P, COLS, A, SECRETS, GAMES = 1024, 32, 4739, 86, 256
POLICY = 150528


def _net(genome_u8: np.ndarray) -> dict:
    h = genome_u8.view(np.float16)[:POLICY + 38 * A].astype(np.float64)
    return dict(We1=h[0:18560].reshape(128, 145), be1=h[18560:18688], We2=h[18688:26880].reshape(64, 128),
                be2=h[26880:26944], W1=h[26944:109120].reshape(256, 321), b1=h[109120:109376],
                W2=h[109376:142144].reshape(128, 256), b2=h[142144:142272], W3=h[142272:150464].reshape(64, 128),
                b3=h[150464:150528], tail=h[POLICY:POLICY + 38 * A].reshape(A, 38))


def _fixed(catalog: np.ndarray) -> np.ndarray:
    counts = np.zeros((len(catalog), 26))
    for p in range(5):
        np.add.at(counts, (np.arange(len(catalog)), catalog[:, p].astype(np.int64)), 1.0)
    return np.where(counts == 0, -1.0, counts)


def _feedback(guess: np.ndarray, secret: np.ndarray) -> np.ndarray:
    """Green pass, then yellows left to right from the secret's unmatched letters (0 green, 1 yellow, 2 grey)."""
    n = len(guess)
    rows = np.arange(n)
    green = guess == secret
    fb = np.where(green, 0, 2).astype(np.uint8)
    counts = np.zeros((n, 26), np.int64)
    for p in range(5):
        m = ~green[:, p]
        np.add.at(counts, (rows[m], secret[m, p].astype(np.int64)), 1)
    for p in range(5):
        letter = guess[:, p].astype(np.int64)
        yellow = ~green[:, p] & (counts[rows, letter] > 0)
        fb[yellow, p] = 1
        counts[rows[yellow], letter[yellow]] -= 1
    return fb


def _forward(net: dict, guesses: np.ndarray, fbs: np.ndarray, turns: np.ndarray) -> np.ndarray:
    """FP64 policy of states given as guesses / feedback [n][5 turns][5] and turn counts [n]."""
    n = len(turns)
    x = np.zeros((n, 321))
    x[:, 0] = turns == 0
    for t in range(5):
        live = turns > t
        if not live.any():
            break
        idx = np.concatenate([np.arange(5) * 26 + guesses[live, t], 130 + np.arange(5) * 3 + fbs[live, t]], axis=1)
        hidden = np.maximum(net["be1"] + net["We1"][:, idx].sum(axis=2).T, 0.0)
        x[live, 1 + 64 * t:65 + 64 * t] = hidden @ net["We2"].T + net["be2"]
    h0 = np.maximum(x @ net["W1"].T + net["b1"], 0.0)
    h1 = np.maximum(h0 @ net["W2"].T + net["b2"], 0.0)
    return h1 @ net["W3"].T + net["b3"]


def _episode(words: np.ndarray, e: int):
    w = len(words)
    s = e // 3
    prefill = [] if e % 3 == 0 else [words[(s + k) % w] for k in ((1, 2) if e % 3 == 1 else (3, 4))]
    return words[s], prefill


def _trace(rt, counts, episodes):
    t = G.torch()
    choices = t.full((P, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((P, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((P, episodes), dtype=t.float32, device="cuda")
    policy = t.zeros((P, episodes, 6, 64), dtype=t.float32, device="cuda")
    rt.evaluate_traced(counts, episodes, choices.data_ptr(), turns.data_ptr(), scores.data_ptr(), policy.data_ptr())
    t.cuda.synchronize()
    return choices.cpu().numpy(), scores.cpu().numpy(), policy.cpu().numpy()


def test_precision_form_against_fp64_host_oracle():
    nwg = G.nwg
    rng = np.random.default_rng(2024)
    catalog = nwg.workload.synthetic_words(A, 3)
    nwg.capi.upload_catalog(catalog)
    subset = nwg.workload.secret_subset(A, 2315, 3)
    offsets, words = nwg.workload.fixed_cell_lists(P, SECRETS, subset, 3)
    rt = nwg.Runtime(A, P, COLS)
    rt.set_cell_words(offsets, words)
    rt.bootstrap(P, seed=3)
    counts = nwg.capi.word_counts(training=A, action_space=A)
    episodes = 3 * SECRETS
    rt.set_form(0)
    plain = _trace(rt, counts, episodes)
    rt.set_form(4)
    rt.set_margin_guard(1e-3)
    form = _trace(rt, counts, episodes)
    slots = rt.current_generation()["slots"]
    genomes = [rt.download_slot(int(s)) for s in slots]
    rt.close()

    # the host Wordle rules against the oracle's
    probe = rng.integers(0, 26, (400, 2, 5)).astype(np.uint8)
    mine = _feedback(probe[:, 0], probe[:, 1])
    assert all(np.array_equal(mine[i], O.feedback(probe[i, 0], probe[i, 1])) for i in range(len(probe)))

    fixed = _fixed(catalog)
    letters = catalog.astype(np.int64)
    pol_err = {"plain": [], "form": []}
    logit_err = []
    raw = {"fp64": np.zeros(P), "plain": plain[1][:, :GAMES].sum(1), "form": form[1][:, :GAMES].sum(1)}
    for i in range(P):
        net = _net(genomes[i])
        emb = np.concatenate([fixed, net["tail"]], axis=1)  # [A][64]
        cell = words[offsets[i]:offsets[i + 1]]
        setup = [_episode(cell, e) for e in range(GAMES)]
        secret = np.array([sec for sec, _ in setup], np.int64)
        # traced decision states of both forms, recomputed in FP64
        for name, (choices, _, policy) in (("plain", plain), ("form", form)):
            seqs = []
            for e, (_, prefill) in enumerate(setup):
                picks = choices[i, e]
                seqs.append(list(prefill) + [int(a) for a in picks[:int((picks >= 0).sum())]])
            flat = np.concatenate([np.array(q, np.int64) for q in seqs])
            fb_flat = _feedback(catalog[flat], catalog[np.repeat(secret, [len(q) for q in seqs])])
            starts = np.concatenate([[0], np.cumsum([len(q) for q in seqs])])
            n_states = sum(len(q) - len(setup[e][1]) for e, q in enumerate(seqs))
            g_arr = np.zeros((n_states, 5, 5), np.int64)
            f_arr = np.zeros((n_states, 5, 5), np.int64)
            n_arr = np.zeros(n_states, np.int64)
            p_arr = np.zeros((n_states, 64))
            k = 0
            for e, q in enumerate(seqs):
                first = len(setup[e][1])
                for step in range(len(q) - first):
                    n = first + step
                    g_arr[k, :n] = letters[q[:n]]
                    f_arr[k, :n] = fb_flat[starts[e]:starts[e] + n]
                    n_arr[k] = n
                    p_arr[k] = policy[i, e, step]
                    k += 1
            p64 = _forward(net, g_arr, f_arr, n_arr)
            pol_err[name].append(np.abs(p_arr - p64).max(1) / np.abs(p64).max(1))
            if name == "form":
                pick = rng.choice(n_states, size=min(24, n_states), replace=False)
                s64 = p64[pick] @ emb.T
                s16 = p_arr[pick].astype(np.float16).astype(np.float64) @ emb.T
                logit_err.append((np.abs(s16 - s64) / s64.std(1, keepdims=True)).ravel())
        # FP64 replay of the 256 games, every live game one guess per round
        hist = np.zeros((GAMES, 6), np.int64)
        fb = np.zeros((GAMES, 6, 5), np.int64)
        n = np.array([len(pf) for _, pf in setup], np.int64)
        for e, (_, prefill) in enumerate(setup):
            if prefill:
                hist[e, :2] = prefill
        pre = np.flatnonzero(n > 0)
        for k in range(2):
            fb[pre, k] = _feedback(catalog[hist[pre, k]], catalog[secret[pre]])
        won = np.zeros(GAMES, bool)
        while True:
            ids = np.flatnonzero(~won & (n < 6))
            if len(ids) == 0:
                break
            scores = _forward(net, letters[hist[ids, :5]], fb[ids, :5], n[ids]) @ emb.T
            for k in range(6):
                m = k < n[ids]
                scores[np.flatnonzero(m), hist[ids[m], k]] = -np.inf
            best = scores.argmax(1)
            hist[ids, n[ids]] = best
            fb[ids, n[ids]] = _feedback(catalog[best], catalog[secret[ids]])
            won[ids] = best == secret[ids]
            n[ids] += 1
        raw["fp64"][i] = float(np.where(won, 10 + 6 - n, 0).sum())

    plain_err = np.concatenate(pol_err["plain"])
    form_err = np.concatenate(pol_err["form"])
    logits = np.concatenate(logit_err)
    scale = 15.0 * GAMES
    summary = {
        "individuals": P, "games_each": GAMES, "actions": A,
        "plain_policy_rel_err": {"max": float(plain_err.max()), "median": float(np.median(plain_err))},
        "form_policy_rel_err": {"max": float(form_err.max()), "p99": float(np.quantile(form_err, 0.99)),
                                "median": float(np.median(form_err))},
        "form_logit_err_over_score_std": {"max": float(logits.max()), "p999": float(np.quantile(logits, 0.999)),
                                          "median": float(np.median(logits)), "samples": int(logits.size)},
        "plain_vs_fp64_fitness": {"identical": int((raw["plain"] == raw["fp64"]).sum()),
                                  "max_delta": float(np.abs(raw["plain"] - raw["fp64"]).max() / scale)},
        "form_vs_fp64_fitness": {"identical": int((raw["form"] == raw["fp64"]).sum()),
                                 "max_delta": float(np.abs(raw["form"] - raw["fp64"]).max() / scale)},
    }
    print("FP64_ORACLE_REPORT " + json.dumps(summary))
    assert plain_err.max() < 1e-4  # the FP32 form is the FP64 recomputation up to FP32 rounding
    assert np.median(form_err) < 5e-3 and np.quantile(form_err, 0.99) < 3e-2
    assert np.quantile(logits, 0.999) < 2e-2
    assert summary["plain_vs_fp64_fitness"]["identical"] >= 0.99 * P
    assert summary["form_vs_fp64_fitness"]["identical"] >= 0.97 * P
