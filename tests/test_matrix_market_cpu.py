"""Matrix Market ingest/export (libuipc_b200.matrix_market, native in
csrc/scene/matrix_market.cpp) against the reference's dump format: the golden
fixture in tests/golden (formatted from the reference's printf formats by
tests/golden/make_golden.py), round trips, and the reader's rules (entries
outside the stated size skipped, blocks ordered by (block row, block column),
a repeated entry keeps the later value). No GPU."""
import json
import os

import numpy as np
import pytest

from libuipc_b200 import matrix_market as mm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden_blocks():
    g = json.load(open(os.path.join(GOLDEN, "mm_blocks.json")))
    rows = np.array([b[0] for b in g["blocks"]], np.int32)
    cols = np.array([b[1] for b in g["blocks"]], np.int32)
    # the fixture lists B row-major; the library keeps 9 values column-major
    vals = np.array([np.array(b[2], np.float64).T.ravel() for b in g["blocks"]])
    return g["n_block_rows"], rows, cols, vals, np.array(g["b"], np.float64)


def test_export_reproduces_the_reference_dump_text(tmp_path):
    nb, rows, cols, vals, b = _golden_blocks()
    a_path, b_path = tmp_path / "A.mtx", tmp_path / "b.mtx"
    mm.export_matrix_market(str(a_path), nb, rows, cols, vals)
    mm.export_vector_market(str(b_path), b)
    assert a_path.read_bytes() == open(os.path.join(GOLDEN, "mm_blocks_A.mtx"), "rb").read()
    assert b_path.read_bytes() == open(os.path.join(GOLDEN, "mm_blocks_b.mtx"), "rb").read()


def test_import_of_the_reference_dump_text():
    nb, rows, cols, vals, b = _golden_blocks()
    nb2, r2, c2, v2 = mm.import_matrix_market(os.path.join(GOLDEN, "mm_blocks_A.mtx"))
    assert nb2 == nb
    np.testing.assert_array_equal(r2, rows)
    np.testing.assert_array_equal(c2, cols)
    assert np.array_equal(v2.view(np.int64), vals.view(np.int64))  # bit-exact, -0.0 included
    x = mm.import_vector_market(os.path.join(GOLDEN, "mm_blocks_b.mtx"))
    assert np.array_equal(x.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("one_based", [True, False])
def test_round_trip_is_bit_exact(tmp_path, one_based):
    rng = np.random.default_rng(7)
    nb = 40
    keys = np.unique(rng.integers(0, nb, size=(300, 2)), axis=0)
    keys = keys[keys[:, 0] <= keys[:, 1]]
    rows, cols = keys[:, 0].astype(np.int32), keys[:, 1].astype(np.int32)
    vals = rng.standard_normal((len(rows), 9)) * 10.0 ** rng.integers(-30, 30, size=(len(rows), 9))
    p = str(tmp_path / "A.mtx")
    mm.export_matrix_market(p, nb, rows, cols, vals, one_based=one_based)
    nb2, r2, c2, v2 = mm.import_matrix_market(p, one_based=one_based)
    assert nb2 == nb
    np.testing.assert_array_equal(r2, rows)
    np.testing.assert_array_equal(c2, cols)
    assert np.array_equal(v2.view(np.int64), vals.view(np.int64))
    x = rng.standard_normal(3 * nb)
    mm.export_vector_market(str(tmp_path / "x.mtx"), x)
    assert np.array_equal(mm.import_vector_market(str(tmp_path / "x.mtx")), x)


def test_reader_rules(tmp_path):
    # unsorted blocks, one entry given twice (the later wins), one outside the
    # stated size (skipped), blank and comment lines between entries
    text = "\n".join([
        "%MatrixMarket matrix coordinate real general",
        "% a comment",
        "6 6 5",
        "4 5 2.0",
        "",
        "1 1 1.5",
        "% another comment",
        "1 1 -3.0",
        "7 1 9.0",
        "2 3 0.25",
    ]) + "\n"
    p = tmp_path / "A.mtx"
    p.write_text(text)
    nb, rows, cols, vals = mm.import_matrix_market(str(p))
    assert nb == 2
    np.testing.assert_array_equal(rows, [0, 1])
    np.testing.assert_array_equal(cols, [0, 1])
    B0 = vals[0].reshape(3, 3).T  # column-major storage -> B[p, q]
    B1 = vals[1].reshape(3, 3).T
    assert B0[0, 0] == -3.0 and B0[1, 2] == 0.25 and np.count_nonzero(B0) == 2
    assert B1[0, 1] == 2.0 and np.count_nonzero(B1) == 1


def test_reader_refusals(tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text("%MatrixMarket matrix coordinate real general\n0 0 0\n")
    with pytest.raises(ValueError):
        mm.import_matrix_market(str(bad))
    vec = tmp_path / "v.mtx"
    vec.write_text("%MatrixMarket matrix array real general\n3 1\n1\n2\n")  # 2 of 3 values
    with pytest.raises(ValueError):
        mm.import_vector_market(str(vec))
    vec.write_text("%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")  # not one column
    with pytest.raises(ValueError):
        mm.import_vector_market(str(vec))
    with pytest.raises(ValueError):
        mm.import_matrix_market(str(tmp_path / "missing.mtx"))


def test_oracle_assembly_survives_a_dump(tmp_path, cube5):
    """The oracle's convert_sym result of a tet cube, dumped and read back,
    is the same block-upper matrix bit for bit."""
    from oracle import oracle as O

    A = O.OracleMatrix(cube5.n_verts, cube5.rows, cube5.cols, cube5.vals)
    rowptr, rows, cols, vals = A.bsr()
    p = str(tmp_path / "A.mtx")
    mm.export_matrix_market(p, cube5.n_verts, rows, cols, vals)
    nb, r2, c2, v2 = mm.import_matrix_market(p)
    assert nb == cube5.n_verts
    np.testing.assert_array_equal(r2, rows)
    np.testing.assert_array_equal(c2, cols)
    assert np.array_equal(v2.view(np.int64), vals.view(np.int64))


def test_golden_metis_partition_of_the_reference():
    """The committed part ids came from the reference's own METIS (compiled
    from its sources); the oracle's partition path reproduces them whenever
    that library is present."""
    from libuipc_b200 import scene
    from oracle import oracle as O

    pid = np.load(os.path.join(GOLDEN, "metis_cube5.npy"))
    cube = scene.cube_on_ground(5, seed=0)
    assert pid.shape == (cube.n_verts,)
    assert np.bincount(pid).max() <= 16
    if not O.metis_available():
        pytest.skip("the reference's METIS build (oracle/_ref) is not present")
    np.testing.assert_array_equal(O.metis_mesh_partition(cube.adj_start, cube.adj_list), pid)
