"""Regenerates tests/golden/hand_constructed.json from the reference's own
fixtures (rivrs-linalg: sparse/test-data/hand-constructed/*.mtx + *.json).

Each entry keeps the matrix (lower-triangle coordinates, as in the .mtx), the
fields the reference's tests assert on (the exact inertia, the D-block sizes)
and the published factorization itself (permutation, strict lower L entries,
D blocks) in the reference's JSON layout (sparse/src/io/reference.rs).

    python tests/golden/make_golden.py /path/to/rivrs-linalg
"""
import json
import os
import sys


def main(ref_root):
    src = os.path.join(ref_root, "sparse", "test-data", "hand-constructed")
    out = {}
    for fn in sorted(os.listdir(src)):
        if not fn.endswith(".mtx"):
            continue
        name = fn[:-4]
        with open(os.path.join(src, fn)) as f:
            header = f.readline().split()
            line = f.readline()
            while line.startswith("%"):
                line = f.readline()
            n, _, nz = (int(x) for x in line.split())
            entries = []
            for _ in range(nz):
                r, c, v = f.readline().split()
                entries.append([int(r) - 1, int(c) - 1, float(v)])
        with open(os.path.join(src, name + ".json")) as f:
            gold = json.load(f)
        out[name] = {
            "n": n,
            "symmetric": "symmetric" in [h.lower() for h in header],
            "entries": entries,
            "inertia": [gold["inertia"]["positive"], gold["inertia"]["negative"], gold["inertia"]["zero"]],
            "d_block_sizes": [b["size"] for b in gold["d_blocks"]],
            # the published factorization itself, in the reference's JSON layout
            "reference": {k: gold[k] for k in ("matrix_name", "permutation", "l_entries", "d_blocks", "inertia")
                          if k in gold},
        }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hand_constructed.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} fixtures to {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/rivrs-linalg")
    main(sys.argv[1])
