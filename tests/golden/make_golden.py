"""Generates the golden fixtures under tests/golden/ (run in a container that
has the reference tree and the compiled reference, oracle/_ref).  The
reference tree is $GPRAT_REFERENCE, else the directory `reference` beside
this repository:

    make -C oracle && python tests/golden/make_golden.py

1. data_1024_n128.json: the reference's own known-answer test
   (test/src/output_correctness.cpp:60-247): the first 128 values of
   data/data_1024/{training_input,training_output,test_input}.txt and the
   expected results of data/data_1024/output.json.
2. ref_cases.npz: outputs of the reference's CPU code (compiled from source,
   oracle/_ref) on seeded synthetic inputs: a 1024-point case with 64-wide
   tiles, a ragged test set, a 64-regressor case, and 5 Adam steps with the
   gradient at every step.
3. c3_optimize.npz (`--c3`, several minutes): the hyper-parameter
   optimisation configuration, n_train = 8192, d = 8, 16 x 16 tiles of 512,
   initial (lengthscale, vertical_lengthscale, noise) = (0.5, 2.0, 0.5),
   50 Adam steps at lr = 0.1: the reference's loss and parameters after every
   step and its gradient at steps 0, 10, 20, 30, 40.
4. ref_large.npz (`--large`, tens of minutes on 8 cores): the benchmark
   configurations at full size, C1 = n_train 16384, n_test 4096, d 8,
   32 x 32 tiles of 512, (1.0, 1.0, 0.1) and C2 = n_train 32768, n_test 8192,
   d 64, 32 x 32 tiles of 1024, (4.0, 1.0, 0.01): predict_with_uncertainty's
   mean and variance, calculate_loss, and of cholesky() the sum and the sum
   of squares of every tile plus three 32 x 32 corners.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import gprat_oracle as O  # noqa: E402
from oracle import ref  # noqa: E402

REF = os.environ.get("GPRAT_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def known_answer():
    d = os.path.join(REF, "data", "data_1024")
    raw = {}
    for name in ("training_input", "training_output", "test_input"):
        raw[name] = np.loadtxt(os.path.join(d, name + ".txt"), max_rows=128).tolist()
    with open(os.path.join(d, "output.json")) as f:
        expected = json.load(f)
    out = {
        "source": "reference data/data_1024 + output.json; config of test/src/output_correctness.cpp:60-71",
        "n_train": 128, "n_test": 128, "n_tiles": 4, "n_reg": 8, "kernel_params": [1.0, 1.0, 0.1],
        "adam": [0.1, 0.9, 0.999, 1e-8, 3],
        "raw": raw,
        "expected": expected,
    }
    with open(os.path.join(HERE, "data_1024_n128.json"), "w") as f:
        json.dump(out, f)


def case_predict(tag, n, m, d, T, hyper, store):
    x, y, xt = O.synthetic(n, m, d)
    nt = n // T
    mt, mts = ref.compute_test_tiles(m, nt, T)
    gp = ref.RefGP(x, y, nt, T, d, hyper)
    mean, var = gp.predict_with_uncertainty(xt, mt, mts)
    fmean, fvar = gp.predict_with_full_cov(xt, mt, mts)
    pmean = gp.predict(xt, mt, mts)
    loss = gp.calculate_loss()
    tiles = gp.cholesky()
    chk = np.array([t.sum() if t is not None else np.nan for t in tiles])
    store.update({
        f"{tag}_cfg": np.array([n, m, d, T, mt, mts], dtype=np.int64),
        f"{tag}_hyper": np.array(hyper),
        f"{tag}_mean": mean, f"{tag}_var": var, f"{tag}_full_mean": fmean, f"{tag}_full_var": fvar,
        f"{tag}_pred": pmean, f"{tag}_loss": np.array([loss]),
        f"{tag}_tile_sums": chk,
        f"{tag}_tile_last": tiles[nt * nt - 1],
        f"{tag}_tile_0": tiles[0],
        f"{tag}_tile_10": tiles[nt],
    })


def case_optimize(store):
    n, d, T = 256, 8, 64
    x, y, _ = O.synthetic(n, 16, d)
    gp = ref.RefGP(x, y, n // T, T, d, (0.5, 2.0, 0.5))
    losses, params, grads = [], [], []
    for it in range(5):
        grads.append(gp.gradient(0.1, 0.9, 0.999, 1e-8))
        losses.append(gp.optimize_step(it, 0.1, 0.9, 0.999, 1e-8))
        params.append(gp.get_params())
    store.update({
        "opt_cfg": np.array([n, d, T], dtype=np.int64),
        "opt_losses": np.array(losses), "opt_params": np.array(params), "opt_grads": np.array(grads),
    })


def case_c3():
    n, d, T, steps = 8192, 8, 512, 50
    adam = (0.1, 0.9, 0.999, 1e-8)
    x, y, _ = O.synthetic(n, 16, d)
    gp = ref.RefGP(x, y, n // T, T, d, (0.5, 2.0, 0.5))
    checkpoints = [0, 10, 20, 30, 40]
    losses, params, grads = [], [], []
    for it in range(steps):
        if it in checkpoints:
            grads.append(gp.gradient(*adam))
        losses.append(gp.optimize_step(it, *adam))
        params.append(gp.get_params())
        print(f"c3 step {it}: loss {losses[-1]:.12f}", flush=True)
    np.savez_compressed(os.path.join(HERE, "c3_optimize.npz"), cfg=np.array([n, d, T, steps], dtype=np.int64),
                        adam=np.array(adam), checkpoints=np.array(checkpoints, dtype=np.int64),
                        losses=np.array(losses), params=np.array(params), grads=np.array(grads))


LARGE = {
    # tag: n, m, d, T, hyper
    "c1": (16384, 4096, 8, 512, (1.0, 1.0, 0.1)),
    "c2": (32768, 8192, 64, 1024, (4.0, 1.0, 0.01)),
}


def case_large(tag, store):
    import time

    n, m, d, T, hyper = LARGE[tag]
    x, y, xt = O.synthetic(n, m, d)
    nt = n // T
    mt, mts = ref.compute_test_tiles(m, nt, T)
    gp = ref.RefGP(x, y, nt, T, d, hyper)
    t0 = time.time()
    mean, var = gp.predict_with_uncertainty(xt, mt, mts)
    t1 = time.time()
    loss = gp.calculate_loss()
    t2 = time.time()
    tiles = gp.cholesky()
    t3 = time.time()
    print(f"{tag}: predict_with_uncertainty {t1 - t0:.1f} s, calculate_loss {t2 - t1:.1f} s, cholesky {t3 - t2:.1f} s",
          flush=True)
    sums = np.array([t.sum() if t is not None else 0.0 for t in tiles])
    sumsq = np.array([np.dot(t, t) if t is not None else 0.0 for t in tiles])
    last = tiles[nt * nt - 1].reshape(T, T)
    store.update({
        f"{tag}_cfg": np.array([n, m, d, T, mt, mts], dtype=np.int64),
        f"{tag}_hyper": np.array(hyper),
        f"{tag}_mean": mean, f"{tag}_var": var, f"{tag}_loss": np.array([loss]),
        f"{tag}_tile_sum": sums, f"{tag}_tile_sumsq": sumsq,
        f"{tag}_corner_00": tiles[0].reshape(T, T)[:32, :32].copy(),
        f"{tag}_corner_last": last[-32:, -32:].copy(),
        f"{tag}_corner_low": tiles[(nt - 1) * nt].reshape(T, T)[:32, :32].copy(),
        f"{tag}_seconds": np.array([t1 - t0, t2 - t1, t3 - t2]),
    })
    del tiles


def main():
    ref.start()
    if "--c3" in sys.argv:
        case_c3()
        return
    if "--large" in sys.argv:
        path = os.path.join(HERE, "ref_large.npz")
        store = dict(np.load(path)) if os.path.exists(path) else {}
        for tag in [a for a in sys.argv[sys.argv.index("--large") + 1:] if a in LARGE] or list(LARGE):
            case_large(tag, store)
            np.savez_compressed(path, **store)
        return
    known_answer()
    store = {}
    case_predict("c0", 1024, 1024, 8, 64, (1.0, 1.0, 0.1), store)
    case_predict("ragged", 256, 200, 8, 64, (1.0, 1.0, 0.1), store)
    case_predict("d64", 512, 256, 64, 128, (4.0, 1.0, 0.01), store)
    case_optimize(store)
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **store)


if __name__ == "__main__":
    main()
