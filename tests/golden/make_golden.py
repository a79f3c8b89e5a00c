"""Generates tests/golden/reference_counts.json by running the reference's own
`tc` and `tc_big_graphs` (compiled unmodified for sm_100a into oracle/_ref by
oracle/Makefile) on seeded synthetic graphs and on the hand-made fixtures.

Needs a GPU (the reference counts only on the GPU). Usage, from the repo
root on a GPU machine:

    python tests/golden/make_golden.py --out tests/golden/reference_counts.json

Each graph is regenerated from its seed by wetric's host generators, written
as a Matrix Market file into a temporary directory, and counted by the
reference with several (s, a) settings; the table rows (n, m, triangles) are
recorded. Bitmap lengths are multiples of 64: for a % 64 == 32 the reference
under-allocates its bitmap (S/32 words, tc.cu:331 and 375).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "wedge-parallel-triangle-counting_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import wetric  # noqa: E402
from wetric import workloads as W  # noqa: E402

# (spec, [(s, a), ...]) -- kept small so every run is seconds.
SEEDED = [
    (W.CHUNG_LU_262K, [(5, 8192), (1, 0), (7, 64)]),
    (W.RmatSpec(scale=10, edge_factor=16, seed=1), [(5, 8192), (1, 0), (3, 64)]),
    (W.RmatSpec(scale=12, edge_factor=16, seed=2), [(5, 8192), (2, 128)]),
    (W.RmatSpec(scale=14, edge_factor=16, seed=3), [(5, 8192), (10, 4096), (1, 0)]),
    (W.RmatSpec(scale=16, edge_factor=16, seed=4), [(5, 8192), (16, 0)]),
    (W.RmatSpec(scale=18, edge_factor=8, seed=5), [(5, 8192)]),
    (W.ErdosRenyiSpec(n=5000, draws=100_000, seed=6), [(5, 8192), (1, 64)]),
    (W.ChungLuSpec(n=20_000, gamma=2.2, i0=8.0, draws=200_000, seed=7), [(5, 8192), (4, 0)]),
    (W.ChungLuSpec(n=100_000, gamma=2.9, i0=40.0, draws=1_200_000, seed=8), [(5, 16384)]),
]


def spec_dict(spec):
    d = dict(kind=type(spec).__name__, name=spec.name)
    d.update({k: getattr(spec, k) for k in spec.__dataclass_fields__})
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    assert oracle.have_reference_binary(), "build oracle/_ref first (make -C oracle ref)"
    out = dict(
        about=("Outputs of the reference's own tc / tc_big_graphs (compiled "
               "unmodified for sm_100a) on seeded graphs and hand fixtures; "
               "made by tests/golden/make_golden.py"),
        seeded=[],
        hand=[],
    )
    with tempfile.TemporaryDirectory() as tmp:
        for spec, settings in SEEDED:
            src, dst, n = W.host_pairs(spec)
            path = os.path.join(tmp, spec.name + ".mtx")
            wetric.write_mm(path, n, src, dst)
            g = oracle.oriented_from_pairs(src, dst)
            maxd = oracle.max_out_degree(g)
            assert maxd < 65536, "reference u32 wedge arithmetic needs d+ < 2^16"
            runs = []
            for s, a in settings:
                for big in (False, True):
                    rows = oracle.run_reference(path, s, a, loops=1, big=big)
                    r = rows[0]
                    runs.append(dict(s=s, a=a, binary="tc_big_graphs" if big else "tc",
                                     n=r["n"], m=r["m"], triangles=r["triangles"],
                                     exec_s=r["exec"]))
            out["seeded"].append(dict(spec=spec_dict(spec), runs=runs))
            print(spec.name, runs[0], flush=True)
    with open(os.path.join(HERE, "hand_graphs.json")) as f:
        hand = json.load(f)
    for h in hand["graphs"] + hand["deviations"]:
        path = os.path.join(HERE, h["file"])
        rows = oracle.run_reference(path, 5, 8192, loops=1, matrix_market=h["mm"],
                                    zero_indexed=h["zero_indexed"])
        r = rows[0]
        out["hand"].append(dict(file=h["file"], n=r["n"], m=r["m"], triangles=r["triangles"]))
        print(h["file"], r["n"], r["m"], r["triangles"], flush=True)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
