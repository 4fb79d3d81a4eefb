"""Generates tests/golden/<case>.npz from the reference's own kernels.

Run on a machine with a B200 and the prebuilt oracle/_ref cubins:
    python tests/golden/make_golden.py
Each file holds the reference's visbuffer (uint64, W*H), its headless RGBA8
image (uint32, W*H) and its stage-2 / stage-3 queue counts, for the seeded
scene of the same name in golden_cases.py.  The reference kernels are the
IEEE-mode build (oracle/build_ref.py): no FMA contraction, IEEE division.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, os.path.join(ROOT, "curast-ooc_b200"), os.path.join(ROOT, "oracle")]

import golden_cases  # noqa: E402
import oracle_lib  # noqa: E402


def make(name, ref):
    c = golden_cases.case(name)
    ref.reset()
    handles = [ref.mesh_host(p, i, col) for (p, i, col) in c["meshes"]]
    ids = [handles[m] for m, _ in c["instances"]]
    worlds = np.stack([np.asarray(w, np.float32).reshape(16) for _, w in c["instances"]])
    vis, cb, rgba, ms, counts = ref.frame(ids, worlds, c["view"], c["proj"], c["W"], c["H"], instanced=True,
                                          display=4, cap_nontrivial=1 << 22, cap_huge=1 << 22)
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, vis=vis, rgba=rgba, counts=counts)
    return out, counts


def main():
    ref = oracle_lib.Reference("ieee")
    for name in golden_cases.CASES:
        out, counts = make(name, ref)
        print(name, "->", os.path.basename(out), "nontrivial", int(counts[0]), "tiles", int(counts[1]))


if __name__ == "__main__":
    main()
