"""Train the learned initial guess on converged FP64 densities and evaluate it.

    python -m rest_b200.train_guess --train 1000 --kmax 12 --epochs 60 \
        --out rest_b200/data/guess_h2o_def2svp.npz --eval 32 --eval-kmin 13 --eval-kmax 24

1. training set: water clusters (H2O)_k with k uniform in [1, kmax] (seeded
   rejection sampling, random orientations), converged by the batched FP64 SCF
   (def2-SVP / def2-SVP-JKFIT, device integrals, Cholesky metric);
2. training: the pair MLP on the device with the library's kernels (masked MSE
   of standardised local density blocks, Adam, cosine learning-rate decay);
3. evaluation on held-out clusters with k in [eval-kmin, eval-kmax]: the same
   batched SCF from REST's hcore guess and from the learned density (with the
   electron-count fallback), reporting iterations, wall time and the energy
   difference.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .geometry import water_cluster
from .guess import LearnedGuess, train
from .sad import sad_density
from .scf_batch import run_molecule_set

BASIS, AUXBAS = "def2-SVP", "def2-SVP-JKFIT"
CRIT = dict(acc_etot=1e-8, acc_rho=1e-6, acc_eev=1e-6, max_cycle=100)


def clusters(count: int, kmin: int, kmax: int, seed: int):
    rng = np.random.default_rng(seed)
    ks = rng.integers(kmin, kmax + 1, count)
    return [water_cluster(int(k), seed=seed * 100003 + i) for i, k in enumerate(ks)]


def evaluate(guess: LearnedGuess, mols, group_size: int = 32) -> dict:
    t0 = time.perf_counter()
    ref = run_molecule_set(mols, BASIS, AUXBAS, group_size=group_size, **CRIT)
    t_ref = time.perf_counter() - t0
    t0 = time.perf_counter()
    lrn = run_molecule_set(mols, BASIS, AUXBAS, group_size=group_size, guess=guess, **CRIT)
    t_lrn = time.perf_counter() - t0
    t_pred = lrn.timings["setup_parts"].get("guess", 0.0)
    fallback = int(lrn.timings["setup_parts"].get("guess_fallbacks", 0))
    # REST's SAD guess (src/initial_guess/sad.rs): atomic SCFs once per element,
    # block-diagonal densities, the first Fock build from them in dm-only form
    t0 = time.perf_counter()
    dens = [sad_density(m, BASIS, AUXBAS)[0] for m in mols]
    t_sad_dens = time.perf_counter() - t0
    sad = run_molecule_set(mols, BASIS, AUXBAS, group_size=group_size, initial_densities=dens, **CRIT)
    t_sad = time.perf_counter() - t0
    de = np.abs(np.array(lrn.energies) - np.array(ref.energies))
    de_sad = np.abs(np.array(sad.energies) - np.array(ref.energies))
    return {
        "molecules": len(mols),
        "hcore": {"iterations_mean": float(np.mean(ref.iterations)), "wall_s": t_ref, "scf_s": ref.scf_s,
                  "converged": int(sum(ref.converged))},
        "sad": {"iterations_mean": float(np.mean(sad.iterations)), "wall_s": t_sad, "scf_s": sad.scf_s,
                "density_s": t_sad_dens, "converged": int(sum(sad.converged)),
                "max_abs_energy_difference_vs_hcore": float(de_sad.max())},
        "learned": {"iterations_mean": float(np.mean(lrn.iterations)), "wall_s": t_lrn, "scf_s": lrn.scf_s,
                    "predict_s": t_pred, "converged": int(sum(lrn.converged)), "fallbacks": int(fallback)},
        "max_abs_energy_difference": float(de.max()),
        "iterations_saved_fraction": float(1.0 - np.mean(lrn.iterations) / np.mean(ref.iterations)),
        "iterations_saved_fraction_vs_sad": float(1.0 - np.mean(lrn.iterations) / np.mean(sad.iterations)),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1000)
    ap.add_argument("--kmax", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default="rest_b200/data/guess_h2o_def2svp.npz")
    ap.add_argument("--eval", type=int, default=32)
    ap.add_argument("--eval-kmin", type=int, default=13)
    ap.add_argument("--eval-kmax", type=int, default=24)
    ap.add_argument("--eval-only", default=None, metavar="WEIGHTS",
                    help="skip training: evaluate the weights in this file")
    a = ap.parse_args()
    if a.eval_only:
        guess = LearnedGuess.load(a.eval_only)
        res = evaluate(guess, clusters(a.eval, a.eval_kmin, a.eval_kmax, a.seed + 7919))
        print(json.dumps({"weights": a.eval_only, "eval": res}), flush=True)
        return
    t0 = time.perf_counter()
    mols = clusters(a.train, 1, a.kmax, a.seed)
    res = run_molecule_set(mols, BASIS, AUXBAS, group_size=64, return_densities=True, **CRIT)
    samples = [(m, d) for m, d, c in zip(mols, res.densities, res.converged) if c]
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    net, norm, hist = train(samples, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    t_train = time.perf_counter() - t0
    guess = LearnedGuess(net, norm, BASIS)
    guess.save(a.out)
    out = {"training_molecules": len(samples), "data_s": t_data, "train_s": t_train, "epochs": a.epochs,
           "loss_first": hist[0], "loss_last": hist[-1], "weights": a.out}
    if a.eval:
        out["eval"] = evaluate(guess, clusters(a.eval, a.eval_kmin, a.eval_kmax, a.seed + 7919))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
