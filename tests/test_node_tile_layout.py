"""Host-side layout of the node-tiled step (ms_node_tile_layout): the same
code and checks ms_create runs before any kernel sees the plan -- CPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import make_model


def _expected(P, N, nt):
    T = P.shape[0]
    K = (N + nt - 1) // nt
    pairs = np.unique(np.stack([np.repeat(np.arange(T), 6), (P // nt).ravel()], 1), axis=0)
    cnt = np.bincount(pairs[:, 1], minlength=K)
    return K, int(cnt.sum()), int(np.maximum(1, -(-cnt // 128)).sum())


@pytest.mark.parametrize("nt", [256, 1024, 4096])
def test_layout_counts(workdir, nt):
    from morphoshell_b200 import MS_PRECISION_MIXED, node_tile_layout
    m = make_model(workdir, "disk18k")
    P = m.tables()["patch_ids"]
    K, pairs, chunks = _expected(P, m.num_nodes, nt)
    for prec in (0, MS_PRECISION_MIXED):
        info = node_tile_layout(P, m.num_nodes, nt, prec)
        assert (info["tiles"], info["tri_tile_pairs"], info["chunks"]) == (K, pairs, chunks)
        fixed = 128 * (6 * 4 + 24 * (4 if prec else 8) + 4 * 8)
        assert info["record_stride"] % 128 == 0
        assert fixed + 16 < info["record_stride"] <= fixed + 16 + 6 * 128 * 6 + 127
        assert info["bytes_per_step"] % 16 == 0
        # The contribution staging area, two node sections and the tile's
        # accumulators (the tables go straight to registers).
        stage = 128 * 18 * (4 if prec else 8)
        assert info["shared_bytes"] == stage + 2 * (info["record_stride"] - fixed) + 24 * nt
    # Border triangles are computed once per tile they touch: the extra work
    # shrinks as tiles grow.
    assert pairs > P.shape[0]


def test_layout_redundancy_shrinks_with_tile_size(workdir):
    from morphoshell_b200 import node_tile_layout
    m = make_model(workdir, "disk18k")
    P = m.tables()["patch_ids"]
    r = [node_tile_layout(P, m.num_nodes, nt)["tri_tile_pairs"] / P.shape[0] - 1 for nt in (256, 512, 1024)]
    assert r[0] > r[1] > r[2] > 0
    assert r[2] < 0.25


def test_layout_rejects_bad_input(workdir):
    from morphoshell_b200 import MsError, node_tile_layout
    m = make_model(workdir, "disk100")
    P = m.tables()["patch_ids"]
    with pytest.raises(MsError):
        node_tile_layout(P, m.num_nodes, 0)
    bad = P.copy()
    bad[3, 2] = m.num_nodes
    with pytest.raises(MsError):
        node_tile_layout(bad, m.num_nodes, 1024)


def test_layout_isolated_node_tile():
    """A tile whose nodes touch no triangle still gets one (empty) chunk."""
    from morphoshell_b200 import node_tile_layout
    P = np.array([[0, 1, 2, 3, 4, 5]], dtype=np.int32)
    info = node_tile_layout(P, 600, 256)
    assert info["tiles"] == 3 and info["chunks"] == 3 and info["tri_tile_pairs"] == 1


def test_layout_repeated_patch_node():
    """A node twice in one patch gives two entries of one run (slot order,
    the order of the node kernel's lists)."""
    from morphoshell_b200 import node_tile_layout
    P = np.array([[0, 1, 2, 0, 1, 2], [1, 2, 3, 0, 4, 5]], dtype=np.int32)
    info = node_tile_layout(P, 6, 256)
    assert info["tiles"] == 1 and info["chunks"] == 1 and info["tri_tile_pairs"] == 2


def test_layout_sliced_order_sizes(workdir):
    """The sliced staging of the warp-specialised step: whole rows of 32
    entries, at least a chunk's entries, and the shared memory of its
    block (two table buffers, two staging areas of three planes, eight node
    sections, the prefetched node state, the accumulators)."""
    from morphoshell_b200 import node_tile_layout
    m = make_model(workdir, "disk18k")
    P = m.tables()["patch_ids"]
    for prec in (0, 1):
        info = node_tile_layout(P, m.num_nodes, 1024, prec)
        slc = info["sliced_entries"]
        assert slc % 32 == 0 and slc >= 6 * 128 // 2
        fixed = 128 * (6 * 4 + 24 * (4 if prec else 8) + 4 * 8)
        stage = -(-3 * slc * (4 if prec else 8) // 128) * 128
        assert info["pipe_shared_bytes"] > 2 * fixed + 2 * stage + 2 * 128 * 8 * 8 + 24 * 1024


def test_layout_same_with_one_thread_and_many(workdir, monkeypatch):
    """The host layout runs one thread per range of tiles; the plan it
    describes does not depend on the thread count."""
    from morphoshell_b200 import MS_PRECISION_MIXED, node_tile_layout
    m = make_model(workdir, "disk18k")
    P = m.tables()["patch_ids"]
    for prec in (0, MS_PRECISION_MIXED):
        monkeypatch.setenv("MORPHOSHELL_SETUP_THREADS", "1")
        one = node_tile_layout(P, m.num_nodes, 300, prec)
        monkeypatch.setenv("MORPHOSHELL_SETUP_THREADS", "7")
        many = node_tile_layout(P, m.num_nodes, 300, prec)
        assert one == many
