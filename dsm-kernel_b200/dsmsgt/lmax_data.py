"""Training data and training runs of the learned angular-order cutoff.

Cutoffs are harvested from the plain method's own runs (dsm_cutoffs: the
banded solves and the device amplitude test, without the l-sum) over
seed-randomised 1-D models, and the network is trained on the GPU by the
library's forward/backward/Adam kernels (dsm_lmax_train).

    python -m dsmsgt.lmax_data --out lmax_params.f32 \\
        --train-seeds 1000:1064 --eval-seeds 2000:2016 --imax 1024

writes the parameter block (DSM_LMAX_NPARAM float32, raw) and prints the
held-out miss rate and padded-work fraction."""
from __future__ import annotations

import argparse
import time

import numpy as np

import dsmsgt
from dsmsgt import synth

MARGIN = 1.02   # the engine's span = predicted cutoff * MARGIN + PAD
PAD = 24.0


def psv_job(seed: int, imax: int, r0: float, tlen: float = 3276.8, rrec: float = 6350.0):
    """P-SV model seed (as in the P-SV configuration), one probe receiver."""
    return dsmsgt.Job(
        synth.param_file(tlen=tlen, rmin=rrec, rmax=rrec, rdelta=100.0, r0=r0, thmin=0.0, thmax=180.0,
                         thdelta=90.0, imin=0, imax=imax),
        synth.dsm_config(), synth.psv_earth_model(seed))


def harvest(seeds, imax: int, depths_km=(10.0, 300.0, 600.0), nfreq: int = 64, tlen: float = 3276.8,
            device: int = 0, log=print):
    """Features and log(llog) for nfreq frequencies spread over 1..imax, for
    every (model seed, source depth)."""
    X, T, G = [], [], []
    freqs = np.unique(np.linspace(1, imax, nfreq).round().astype(int))
    for sd in seeds:
        for dep in depths_km:
            t0 = time.perf_counter()
            s = dsmsgt.Setup(psv_job(sd, imax, 6371.0 - dep, tlen), "psv")
            ctx = dsmsgt.Context(s, device=device, freq_batch=16)
            ll = ctx.cutoffs(freqs)
            f = ctx.lmax_features(freqs)
            X.append(f)
            # target: the cutoff relative to the lsuf scale exp(f0)
            T.append((np.log(np.maximum(ll, 1)) - f[:, 0]).astype(np.float32))
            G.append(np.full(len(freqs), sd))
            ctx.close()
            log(f"seed {sd} depth {dep} km: cutoffs {ll.min()}..{ll.max()} ({time.perf_counter() - t0:.1f} s)")
    return np.concatenate(X), np.concatenate(T), np.concatenate(G)


def plain_ranges(first: int, llog: int, maxl: int = 80000):
    """Orders solved and rounds taken by the plain schedule: a first range,
    then ranges growing by half until the cutoff is inside."""
    solved, span, rounds = 0, first, 0
    while True:
        solved += span
        rounds += 1
        if solved > llog or solved > maxl:
            return solved, rounds
        span = min(4096, span + span // 2)


def evaluate(params, seeds, imax: int, depths_km=(10.0, 300.0, 600.0), nfreq: int = 64, tlen: float = 3276.8,
             device: int = 0):
    """Held-out comparison of the learned first range with the plain one:
    miss rate (first range short of the cutoff, so the device test extends
    it), orders solved beyond the cutoff, and solve rounds."""
    freqs = np.unique(np.linspace(1, imax, nfreq).round().astype(int))
    rows = []
    for sd in seeds:
        for dep in depths_km:
            s = dsmsgt.Setup(psv_job(sd, imax, 6371.0 - dep, tlen), "psv")
            ctx = dsmsgt.Context(s, device=device, freq_batch=16, use_lmax_predictor=1)
            ctx.set_lmax_model(params)
            ll = ctx.cutoffs(freqs)
            pl = ctx.lmax_predict(freqs)
            f = ctx.lmax_features(freqs)
            ctx.close()
            lsuf = (np.expm1(f[:, 0].astype(np.float64)) - 0.5).astype(np.int64) + 1
            for k, i in enumerate(freqs):
                learned = int(np.ceil(max(np.exp(pl[k]) * MARGIN + PAD, lsuf[k] + 8) / 32) * 32)
                plain = int(np.ceil(max(512, lsuf[k] + 64) / 32) * 32)
                ls, lr = plain_ranges(learned, int(ll[k]))
                ps, pr = plain_ranges(plain, int(ll[k]))
                rows.append((int(ll[k]), learned, ls, lr, ps, pr))
    r = np.array(rows, dtype=np.float64)
    used = r[:, 0].sum()
    return {"n": len(r), "miss_rate": float(np.mean(r[:, 1] <= r[:, 0])),
            "padded_learned": float((r[:, 2] - r[:, 0]).sum() / used),
            "padded_plain": float((r[:, 4] - r[:, 0]).sum() / used),
            "rounds_learned": float(r[:, 3].mean()), "rounds_plain": float(r[:, 5].mean()),
            "median_abs_log_err": float(np.median(np.abs(np.log(r[:, 1] / MARGIN) - np.log(r[:, 0]))))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--train-seeds", default="1000:1064")
    ap.add_argument("--eval-seeds", default="2000:2016")
    ap.add_argument("--weight-decay", type=float, default=1e-3)
    ap.add_argument("--imax", type=int, default=2048)
    ap.add_argument("--nfreq", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    a = ap.parse_args()
    lo, hi = (int(v) for v in a.train_seeds.split(":"))
    X, T, _ = harvest(range(lo, hi), a.imax, nfreq=a.nfreq)
    P = dsmsgt.lmax_init(X, T, seed=0)
    P, losses = dsmsgt.lmax_train(X, T, P, epochs=a.epochs, batch=a.batch, lr=a.lr, weight_decay=a.weight_decay)
    print(f"loss {losses[0]:.4f} -> {losses[-1]:.5f} on {len(T)} cutoffs")
    P.astype(np.float32).tofile(a.out)
    lo, hi = (int(v) for v in a.eval_seeds.split(":"))
    print("held-out", evaluate(P, range(lo, hi), a.imax, nfreq=a.nfreq))
    print("benchmark model (seed 0)", evaluate(P, [0], a.imax, depths_km=(300.0,), nfreq=a.nfreq))


if __name__ == "__main__":
    main()
