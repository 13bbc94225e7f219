"""Writes tests/golden/meshio/: a selection of the reader test cases and, in
expected.json, what the reference viewer's reader (viewer/mesh_io.cpp, built
into oracle/_ref/libmeshio_ref.so by oracle/Makefile) returns for each: vertex
bits (hex), faces, error text.  Run from the repository root with the
reference tree present:  python tests/golden/make_meshio_golden.py"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

import meshio_cases as mc  # noqa: E402
import oracle  # noqa: E402

PICK = ["plain.xyz", "comments.xyz", "crlf.txt", "spaces.pts", "numbers.xyz", "bad_numbers.xyz",
        "quad.obj", "negative.obj", "bad_faces.obj", "tags.obj", "cube.off", "counts_on_magic.off",
        "coff.off", "split_counts.off", "truncated.off", "bad_faces.off", "ascii.ply", "crlf.ply",
        "order.ply", "edges.ply", "short_rows.ply", "early_end.ply", "binary.ply", "binary_truncated.ply",
        "binary.stl", "binary_solid_header.stl", "ascii.stl", "ascii_degenerate.stl", "unknown.abc"]


def main():
    out_dir = os.path.join(HERE, "meshio")
    os.makedirs(out_dir, exist_ok=True)
    cases = mc.hand_cases()
    rnd = mc.random_cases(n_each=2, seed=11)
    chosen = {k: cases[k] for k in PICK}
    chosen.update(rnd)
    expected = {}
    for name, data in chosen.items():
        path = os.path.join(out_dir, name)
        with open(path, "wb") as fh:
            fh.write(data)
        v, f, err = oracle.ref_mesh_load(path)
        expected[name] = {"error": err,
                          "vertex_bits": [format(int(x), "016x") for x in v.reshape(-1).view(np.uint64)],
                          "faces": f.reshape(-1).tolist()}
    with open(os.path.join(out_dir, "expected.json"), "w") as fh:
        json.dump(expected, fh, indent=0, sort_keys=True)
    print(f"{len(expected)} cases in {out_dir}")


if __name__ == "__main__":
    main()
