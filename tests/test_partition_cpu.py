"""The graph partitioner (b2s_partition_graph), the library's drop-in for
geometry::mesh_partition's METIS k-way call (src/geometry/mesh_partition.cpp:
77-231), on the CPU: the reference's contract (ceil(n / 16) parts of at most
16 vertices, contiguous non-empty ids, sequential blocks for point clouds,
connected components for n <= 16), determinism, and quality against the
reference's own METIS partitions (tests/golden/metis_*.npy: a cube, a bar, and
three stacked cubes joined by contact pairs): edge cut and the oracle's MAS-PCG
iteration count within 15 % of METIS's."""
import os

import numpy as np
import pytest

from libuipc_b200 import scene
from libuipc_b200.linear_system import B200SolveError, partition_graph, partition_maps
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cut(s, pid):
    src = np.repeat(np.arange(s.n_verts), np.diff(s.adj_start))
    return int((pid[src] != pid[s.adj_list]).sum() // 2)


def _check_contract(n, pid, max_part=16):
    assert pid.shape == (n,) and pid.min() == 0
    counts = np.bincount(pid)
    assert counts.size == (n + max_part - 1) // max_part
    assert counts.max() <= max_part and counts.min() >= 1


def _mas_iterations(s, pid):
    p2r, r2p = partition_maps(pid)
    A = O.OracleMatrix(s.n_verts, s.rows, s.cols, s.vals)
    M = O.OracleMAS(s.n_verts, s.adj_start, s.adj_list, p2r, r2p)
    M.assemble(A, 0, 1)
    _, info = O.pcg(A, s.b, precond=O.ORC_PRECOND_MAS, mas=M, tol=1e-4, stop_rule=O.ORC_STOP_RELRES, threads=1)
    assert info["converged"] == 1
    return info["iterations"]


@pytest.mark.parametrize("mesh", ["cube10", "stack_small", "bar"])
def test_contract_and_determinism(request, mesh):
    s = scene.twisted_bar(30, 4, 4) if mesh == "bar" else request.getfixturevalue(mesh)
    pid = partition_graph(s.adj_start, s.adj_list)
    _check_contract(s.n_verts, pid)
    assert np.array_equal(pid, partition_graph(s.adj_start, s.adj_list))
    # most parts are connected pieces of the mesh
    connected = 0
    for p in range(pid.max() + 1):
        vs = np.flatnonzero(pid == p)
        seen = {vs[0]}
        todo = [vs[0]]
        while todo:
            v = todo.pop()
            for u in s.adj_list[s.adj_start[v]:s.adj_start[v + 1]]:
                if pid[u] == p and u not in seen:
                    seen.add(u)
                    todo.append(u)
        connected += len(seen) == vs.size
    assert connected >= 0.9 * (pid.max() + 1)


@pytest.mark.parametrize("name, make", [
    ("metis_cube10.npy", lambda: scene.cube_on_ground(10, seed=0)),
    ("metis_bar60.npy", lambda: scene.twisted_bar(60, 8, 8)),
    ("metis_stack3x8.npy", lambda: scene.stacked_cubes(8, 3, seed=0)),
])
def test_quality_against_the_reference_metis(name, make):
    s = make()
    ref = np.load(os.path.join(GOLDEN, name)).astype(np.int32)
    assert ref.size == s.n_verts and np.bincount(ref).max() <= 16
    pid = partition_graph(s.adj_start, s.adj_list)
    _check_contract(s.n_verts, pid)
    assert _cut(s, pid) <= 1.15 * _cut(s, ref)
    assert _mas_iterations(s, pid) <= 1.15 * _mas_iterations(s, ref)


def test_point_cloud_and_small_inputs():
    # no edges: sequential blocks of 16, as the reference's point-cloud branch
    n = 40
    pid = partition_graph(np.zeros(n + 1, np.int32), np.zeros(0, np.int32))
    assert np.array_equal(pid, np.arange(n) // 16)
    # n <= 16: one part per connected component (two paths 0-1-2 and 3-4, 5 alone)
    edges = {0: [1], 1: [0, 2], 2: [1], 3: [4], 4: [3], 5: []}
    start = np.cumsum([0] + [len(edges[v]) for v in range(6)]).astype(np.int32)
    lst = np.array([u for v in range(6) for u in edges[v]], np.int32)
    assert list(partition_graph(start, lst)) == [0, 0, 0, 1, 1, 2]
    # empty input
    assert partition_graph(np.zeros(1, np.int32), np.zeros(0, np.int32)).size == 0


def test_disconnected_pieces_stay_within_the_contract():
    """Two meshes with no edge between them (cubes of 5^3 cells, 216
    vertices each, 432 in all): 27 parts of at most 16, and no part mixes the
    two pieces except where a piece's vertex count is not a multiple of 16."""
    c = scene.cube_on_ground(5, seed=0)
    n = c.n_verts
    start = np.concatenate([c.adj_start, c.adj_start[1:] + c.adj_start[-1]]).astype(np.int32)
    lst = np.concatenate([c.adj_list, c.adj_list + n]).astype(np.int32)
    pid = partition_graph(start, lst)
    _check_contract(2 * n, pid)
    mixed = sum(1 for p in range(pid.max() + 1) if len({int(v >= n) for v in np.flatnonzero(pid == p)}) > 1)
    assert mixed <= 1


def test_invalid_adjacency_is_an_argument_error():
    start = np.array([0, 1, 2], np.int32)
    with pytest.raises(B200SolveError):
        partition_graph(start, np.array([1, 5], np.int32))  # neighbour 5 of a 2-vertex graph
    with pytest.raises(B200SolveError):
        partition_graph(np.array([0, 2, 1], np.int32), np.array([1, 0], np.int32))  # decreasing offsets
