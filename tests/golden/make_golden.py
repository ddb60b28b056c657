"""Generates the committed parity fixtures in tests/golden/ (run in the build
container, where the reference tree is readable).

* ref_inputs.npz: the reference's own input fixtures (input/bird.txt,
  input/alpha.txt, input/1000_1.txt, input/10000_1.txt), parsed with the
  reference's reader format (main.cu:117-161: N, then 'index x y').  These are
  the only inputs the reference ships; it ships no outputs.
* golden_<name>.npz: the CPU oracle's exact Delaunay triangulation (canonical
  vertex triples) and alpha output for each input and for config c1, pinned by
  the exact checkResult invariants (main.cu:163-343) in tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from galpha_b200 import datasets as D  # noqa: E402
from galpha_b200.api import read_points_file  # noqa: E402

# the reference tree (read only for its input/ fixtures); GALPHA_REF_TREE overrides
REF_TREE = os.environ.get("GALPHA_REF_TREE", "/root/reference")
REF_INPUT = os.path.join(REF_TREE, "input")
NAMES = ["bird", "alpha", "1000_1", "10000_1"]


def canon(v):
    v = np.asarray(v, dtype=np.int64)
    r = np.argmin(v, axis=1)
    rows = np.arange(len(v))
    c = np.stack([v[rows, (r + k) % 3] for k in range(3)], axis=1)
    return c[np.lexsort((c[:, 2], c[:, 1], c[:, 0]))].astype(np.int32)


def main():
    inputs = {}
    if os.path.isdir(REF_INPUT):
        for nm in NAMES:
            inputs["ref_" + nm] = read_points_file(os.path.join(REF_INPUT, nm + ".txt"))
        np.savez_compressed(os.path.join(HERE, "ref_inputs.npz"), **inputs)
    else:
        z = np.load(os.path.join(HERE, "ref_inputs.npz"))
        inputs = {k: z[k] for k in z.files}
    inputs["c1"] = D.make("c1")[0]
    for nm, pts in inputs.items():
        v, n, kept = O.dt(pts)
        a = O.alpha(pts, v, n)
        # alpha keyed canonically (independent of triangle order)
        tri_key = canon(v)
        tri_rank = {tuple(sorted(map(int, t))): int(r) for t, r in zip(v, a["tri_ro"])}
        tri_ro = np.array([tri_rank[tuple(sorted(map(int, t)))] for t in tri_key], dtype=np.int32)
        E = a["edge"]
        ek = np.stack([np.minimum(E[:, 0], E[:, 1]), np.maximum(E[:, 0], E[:, 1])], axis=1)
        order = np.lexsort((ek[:, 1], ek[:, 0]))
        np.savez_compressed(
            os.path.join(HERE, "golden_%s.npz" % nm),
            points=pts, triangles=tri_key, nkept=kept,
            spectrum=a["spectrum"], tri_ro=tri_ro,
            edge_key=ek[order].astype(np.int32), edge_ranks=E[order][:, 2:5].astype(np.int32),
            point=a["point"],
        )
        print(nm, len(pts), "points", len(v), "triangles", len(a["spectrum"]), "spectrum")


if __name__ == "__main__":
    main()
