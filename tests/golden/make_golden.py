"""Writes the golden fixtures of tests/golden (run from the repository root:
``python tests/golden/make_golden.py``).

* ``mm_blocks_A.mtx``, ``mm_blocks_b.mtx``: a 2-block-row system in the exact
  text the reference's debug dump produces, formatted here in Python from the
  reference's printf formats (src/backends/cuda/utils/matrix_market.h:102-109
  header and dimension lines, :88 entry line "{} {} {:.17g}", :143-153 vector
  lines "%.17g"; the banner comes out with one '%', since a printf-style
  format turns "%%" into "%"), independently of the library's C++ writer; the
  blocks are listed in ``mm_blocks.json``.
* ``metis_cube5.npy``: the part id of every vertex of the 5^3-cell jittered
  tet cube (seed 0) from the reference's own vendored METIS 5.2.1
  (src/geometry/metis, compiled from those sources into oracle/_ref by
  oracle/build_oracle.py) through the oracle's restatement of
  geometry::mesh_partition (seed 0, parts of at most 16 vertices). Needs the
  reference sources (the oracle build), so it is generated here and committed.
* ``metis_cube10.npy``, ``metis_bar60.npy``, ``metis_stack3x8.npy``: the same
  for the 10^3-cell jittered cube (seed 0), the 60x8x8-cell twisted bar and
  three stacked 8^3-cell cubes (seed 0, the stack's first Newton system: a
  mesh of several bodies joined by contact pairs) -- the reference partitions
  of the graph partitioner's quality checks.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# block row, block column, 3x3 value (row-major here); values exercise %.17g
BLOCKS = [
    (0, 0, [[4.0, 0.1, 0.0], [0.1, 5.5, -1e-300], [0.0, -1e-300, 1.0 / 3.0]]),
    (0, 1, [[-1.0, 0.0, 2.5e-8], [0.0, 3.0000000000000004, 0.0], [7.0, -0.0, 1e+22]]),
    (1, 1, [[2.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 123456789.123456789]]),
]
B_VEC = [1.0, -0.5, 0.1, 1e-17, 2.0 / 3.0, -123.25]


def matrix_text(n_block_rows: int, blocks) -> str:
    dim = 3 * n_block_rows
    nnz = 9 * len(blocks)
    out = [
        "%MatrixMarket matrix coordinate real general\n",
        "% Exported from block-sparse triplet matrix\n",
        "% Block dimension: 3x3\n",
        f"% Total rows: {dim}, Total cols: {dim}\n",
        f"% Total entries (including zeros): {nnz}\n",
        f"{dim} {dim} {nnz}\n",
    ]
    for bi, bj, m in blocks:
        for p in range(3):
            for q in range(3):
                out.append("%d %d %.17g\n" % (3 * bi + p + 1, 3 * bj + q + 1, m[p][q]))
    return "".join(out)


def vector_text(x) -> str:
    out = ["%MatrixMarket matrix array real general\n", "% Exported from dense vector\n",
           f"% Vector size: {len(x)}\n", f"{len(x)} 1\n"]
    out += ["%.17g\n" % v for v in x]
    return "".join(out)


def main() -> None:
    with open(os.path.join(HERE, "mm_blocks_A.mtx"), "w") as f:
        f.write(matrix_text(2, BLOCKS))
    with open(os.path.join(HERE, "mm_blocks_b.mtx"), "w") as f:
        f.write(vector_text(B_VEC))
    with open(os.path.join(HERE, "mm_blocks.json"), "w") as f:
        json.dump({"n_block_rows": 2, "blocks": [[bi, bj, m] for bi, bj, m in BLOCKS], "b": B_VEC}, f, indent=1)
    sys.path.insert(0, ROOT)
    from libuipc_b200 import scene
    from oracle import build_oracle
    from oracle import oracle as O

    build_oracle.build_oracle_lib()
    cube = scene.cube_on_ground(5, seed=0)
    pid = O.metis_mesh_partition(cube.adj_start, cube.adj_list)
    np.save(os.path.join(HERE, "metis_cube5.npy"), pid.astype(np.int32))
    for name, mesh in (("metis_cube10.npy", scene.cube_on_ground(10, seed=0)),
                       ("metis_bar60.npy", scene.twisted_bar(60, 8, 8)),
                       ("metis_stack3x8.npy", scene.stacked_cubes(8, 3, seed=0))):
        pid = O.metis_mesh_partition(mesh.adj_start, mesh.adj_list)
        np.save(os.path.join(HERE, name), pid.astype(np.int16))


if __name__ == "__main__":
    main()
