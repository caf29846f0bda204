"""Generate tests/golden/det_batch.npz from the reference core.

Run in a container that has the reference tree (the recipe compiles it from
its own sources into oracle/_ref/):

    make -C oracle ref && python tests/golden/make_det_batch.py

The fixture holds seeded determinant batches with the reference's
prepare_det_batch outputs (det_batch.cpp:184-318, called as its nanobind
bridge does, bridge.cpp:347-430) for every combination of requested fields,
and the reference's message for each invalid call in ERROR_CASES.
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle import Checker  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "det_batch.npz")

# (n_orb, n_alpha, n_beta, kmax, batch size, seed)
CASES = [(8, 3, 3, 4, 64, 1), (13, 5, 5, 2, 64, 2), (30, 12, 12, 8, 96, 3),
         (64, 20, 17, 6, 64, 4), (64, 32, 32, 40, 32, 5), (5, 0, 2, 3, 16, 6)]
# (need_k, need_phase, need_hp, need_hp_pos)
FLAGS = [(False, False, False, False), (True, True, False, False),
         (False, True, True, False), (True, True, True, True)]
ERROR_CASES = [
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=65, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=2, need_hp_pos=True),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=-1, need_hp=True),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=2, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7]], ref=[7, 7], n_orb=4, n_alpha=2, n_beta=3),
    dict(dets=[[7, 7]], ref=[3, 7], n_orb=4, n_alpha=3, n_beta=3, need_phase=True),
    dict(dets=[[7, 7]], ref=[3, 7], n_orb=4, n_alpha=3, n_beta=3, kmax=2, need_hp=True,
         need_hp_pos=True),
    dict(dets=[[7, 7], [15, 7], [16, 7]], ref=[7, 7], n_orb=4, n_alpha=3, n_beta=3),
    dict(dets=[[7, 7], [7, 7], [0b1011, 0b10111]], ref=[7, 7], n_orb=5, n_alpha=3, n_beta=3),
]


def random_dets(rng, n_orb, na, nb, B):
    out = np.zeros((B, 2), np.uint64)
    for i in range(B):
        for s, ne in ((0, na), (1, nb)):
            for o in rng.choice(n_orb, ne, replace=False):
                out[i, s] |= np.uint64(1) << np.uint64(o)
    return out


def main() -> None:
    ref = Checker.reference()
    out = {}
    for c, (n_orb, na, nb, kmax, B, seed) in enumerate(CASES):
        rng = np.random.default_rng(seed)
        r = random_dets(rng, n_orb, na, nb, 1)[0]
        d = random_dets(rng, n_orb, na, nb, B)
        d[0] = r   # the reference itself: k = 0
        out[f"c{c}_dets"] = d
        out[f"c{c}_ref"] = r
        out[f"c{c}_shape"] = np.array([n_orb, na, nb, kmax], np.int64)
        for f, fl in enumerate(FLAGS):
            res = ref.prepare_det_batch(d, r, n_orb, na, nb, kmax, *fl)
            for k, v in res.items():
                out[f"c{c}_f{f}_{k}"] = v
    msgs = []
    for e in ERROR_CASES:
        e = dict(e)
        e["dets"] = np.array(e["dets"], np.uint64)
        try:
            ref.prepare_det_batch(**e)
            msgs.append("")
        except ValueError as err:
            msgs.append(str(err))
    out["error_messages"] = np.array(msgs)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(CASES)} batches x {len(FLAGS)} field sets, {len(msgs)} errors")


if __name__ == "__main__":
    main()
