"""Generate tests/golden/settle_pile_f64.npz: a long run of the oracle.

    python tests/golden/make_golden_settle.py [STEPS]

Runs the oracle's FP64 CUDA scheme (oracle/ps_oracle.c) on the 4,096-sphere
settling pile (psb200.scenes.settle_pile) for STEPS steps (default 40,000,
about three minutes on one core) and records the SHA-256 of the final state
and its settling statistics: the packing fraction of the slab
z in [0.02, 0.16], the height histogram of the sphere centres (24 bins over
[0, 0.3]), the mean centre height and the kinetic energy.  The GPU long-run
test checks its FP64 run bit for bit through the hash and its FP32 run and
the reference CUDA build against the statistics.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "particle-stabilizer_b200", "python"))

from oracle import ps_oracle as O  # noqa: E402
from psb200 import scenes  # noqa: E402

SLAB = (0.02, 0.16)
HIST_TOP = 0.3
HIST_BINS = 24


def summary(sc, state: np.ndarray) -> dict:
    return {
        "packing": scenes.slab_packing_fraction(state, sc.box_min, sc.box_max, *SLAB),
        "hist": scenes.height_histogram(state, HIST_TOP, HIST_BINS),
        "zmean": float(np.mean(state[:, 2])),
        "ke": float(O.stats(np.ascontiguousarray(state, dtype=np.float64)).kinetic_energy),
    }


def state_hash(state: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(state, dtype=np.float64).tobytes()).hexdigest()


def main() -> None:
    steps = int(sys.argv[1]) if len(sys.argv) > 1 else 40000
    sc = scenes.settle_pile()
    final = O.run(sc, steps, "f64")
    s = summary(sc, final)
    out = os.path.join(HERE, "settle_pile_f64.npz")
    np.savez(out, steps=steps, sha256=state_hash(final), packing=s["packing"], hist=s["hist"], zmean=s["zmean"],
             ke=s["ke"], slab=np.array(SLAB), hist_top=HIST_TOP)
    print(out, steps, s["packing"], s["zmean"], s["ke"])


if __name__ == "__main__":
    main()
