"""v_xc checkpoint round trips in the reference's text format (CPU)."""
import numpy as np
import pytest

from conftest import problem


def test_write_read_round_trip(tmp_path):
    from invdft_b200.checkpoint import read_vxc, write_vxc
    P = problem("tiny_h2")
    v = np.random.default_rng(1).standard_normal(P.n_child_nodes)
    f = tmp_path / "vxc_0"
    write_vxc(f, P.child_node_xyz, v)
    assert np.array_equal(read_vxc(f, P.child_node_xyz), v)
    first = f.read_text().splitlines()[0].split()
    assert len(first) == 5 and first[0] == "0"


def test_search_reader_handles_permuted_rows(tmp_path):
    from invdft_b200.checkpoint import read_vxc
    P = problem("tiny_h2")
    v = np.random.default_rng(2).standard_normal(P.n_child_nodes)
    perm = np.random.default_rng(3).permutation(P.n_child_nodes)
    f = tmp_path / "vxc_perm"
    np.savetxt(f, np.column_stack([perm, P.child_node_xyz[perm] + 1e-5, v[perm]]))
    assert np.allclose(read_vxc(f, P.child_node_xyz, search=True), v)
    with pytest.raises(ValueError):
        read_vxc(f, P.child_node_xyz + 0.5, search=True)


def test_coordinate_mismatch_is_an_error(tmp_path):
    from invdft_b200.checkpoint import read_vxc, write_vxc
    P = problem("tiny_h2")
    f = tmp_path / "vxc_bad"
    write_vxc(f, P.child_node_xyz + 0.01, np.zeros(P.n_child_nodes))
    with pytest.raises(ValueError):
        read_vxc(f, P.child_node_xyz)


def test_ordered_reader_places_by_row_position(tmp_path):
    """readVxcDataFromFile (InverseDFTEngine.cpp:2935-2975) checks row i against
    node i and stores row i at node i; a duplicated iNode column does not move
    values, and a column outside [0, n) is rejected."""
    from invdft_b200.checkpoint import read_vxc
    P = problem("tiny_h2")
    n = P.n_child_nodes
    v = np.random.default_rng(4).standard_normal(n)
    ids = np.arange(n)
    ids[1] = 0                                   # duplicated id
    f = tmp_path / "vxc_dup"
    np.savetxt(f, np.column_stack([ids, P.child_node_xyz, v]))
    assert np.array_equal(read_vxc(f, P.child_node_xyz), np.loadtxt(f)[:, 4])
    ids[2] = n + 5
    np.savetxt(f, np.column_stack([ids, P.child_node_xyz, v]))
    with pytest.raises(ValueError):
        read_vxc(f, P.child_node_xyz)
