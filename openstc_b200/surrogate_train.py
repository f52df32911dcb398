"""Train the chemistry surrogate on a data set of FP64 EPI labels and report
its held-out accuracy.

    python -m openstc_b200.surrogate_train CASE_DIR [--samples 16M] [--held-out 1M]
        [--steps 8000] [--batch 65536] [--lr 2e-3] [--field-fraction 0.5]
        [--snapshot-steps 5] [--out surrogate.bin] [--report report.json]

The samples blend the case's flow field (after --snapshot-steps steps of the
FP32-bulk solver; each cell's T and p perturbed by 2 %, its mass fractions by
a log-normal factor, its own local time step within a factor of 2) with
uniform draws from the training box (T in [250, 2800] K, log10 p in [4.5, 6],
Dirichlet(1) mass fractions, log10 dt in [-9, -6]); each is labelled with the
increment of one FP64 point-implicit (EPI) chemistry step at fixed density.
The network trains on the first --samples and is judged on the --held-out
samples after them: max and mean relative dY error and the element defect of
the applied prediction, over the samples the trust gate accepts, plus the
median and 90th percentile of the error over every held-out sample.
"""
from __future__ import annotations

import argparse
import json
import time

import openstc_b200 as ostc


def count(text: str) -> int:
    text = text.strip().upper()
    scale = {"K": 1 << 10, "M": 1 << 20}.get(text[-1:], 1)
    return int(float(text[:-1] if scale > 1 else text) * scale)


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case")
    ap.add_argument("--samples", default="16M")
    ap.add_argument("--held-out", default="1M")
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--field-fraction", type=float, default=0.5)
    ap.add_argument("--snapshot-steps", type=int, default=5)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    n_train, n_held = count(a.samples), count(a.held_out)

    drv = ostc.Driver(a.case, precision="mixed")
    drv.initialize()
    drv.step(a.snapshot_steps)
    sur = ostc.Surrogate(drv, seed=a.seed)
    t0 = time.perf_counter()
    sur.generate(n_train + n_held, seed=a.seed + 1, field=drv, field_fraction=a.field_fraction)
    t1 = time.perf_counter()
    losses = sur.train(a.steps, batch=a.batch, lr=a.lr, n_train=n_train)
    t2 = time.perf_counter()
    held = sur.evaluate(n_train, n_held)
    report = {
        "samples": n_train, "held_out": n_held, "batch": a.batch, "steps": a.steps, "lr": a.lr,
        "epochs": a.steps * a.batch / n_train, "field_fraction": a.field_fraction,
        "generate_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2),
        "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
        "held_out_stats": held, "gate": sur.gate(),
    }
    if a.out:
        sur.save(a.out)
    text = json.dumps(report, indent=1)
    if a.report:
        with open(a.report, "w") as f:
            f.write(text + "\n")
    print(text)
    sur.close()
    drv.close()
    return report


if __name__ == "__main__":
    main()
