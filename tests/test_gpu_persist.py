"""Saved and reloaded trees answer exactly like the trees they came from; a
damaged file is refused at load time (before any query reads it)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HEADER = 216           # bytes of the stored header
HASH_AT = 208          # offset of its checksum field
SECTIONS_AT = 144      # offset of its eight section sizes


def _fnv_words(b):
    """The stored checksum: FNV-1a over 8-byte little-endian words, then
    the tail bytes."""
    h = 1469598103934665603
    n8 = len(b) // 8 * 8
    for w in np.frombuffer(b[:n8], dtype="<u8").tolist():
        h = ((h ^ w) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    for c in b[n8:]:
        h = ((h ^ c) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_tree_round_trip(gpu, tmp_path):
    from pptk_b200 import _native as N
    kd = gpu.kdtree
    rng = np.random.default_rng(0)
    P = rng.random((60_000, 3)).astype(np.float32)
    P[::101] = np.nan  # dropped rows survive the round trip
    t = kd._build(P)
    t.set_bucket(32)
    path = tmp_path / "tree.bin"
    t.save(path)
    u = kd.load(path)
    assert (u.n, u.n_valid, u.dim, u.dtype) == (t.n, t.n_valid, t.dim, t.dtype)
    assert np.array_equal(u.reverse_indices(), t.reverse_indices())
    assert np.array_equal(u.ref_nodes(), t.ref_nodes())
    q = rng.random((5000, 3)).astype(np.float32)
    for a, b in zip(kd.knn(u, q, 12), kd.knn(t, q, 12)):
        assert np.array_equal(a, b)
    for a, b in zip(kd.rnear(u, q[:500], 0.02), kd.rnear(t, q[:500], 0.02)):
        assert np.array_equal(a, b)
    ev = [np.empty((len(P), 3), np.float32) for _ in range(2)]
    for tree, out in zip((t, u), ev):
        N.call("pptkg_tree_normals", tree._h, None, 0, N.MEM_HOST, 10, ctypes.c_float(np.inf), 1, 0, N.ptr(out), None,
               None, None)
    assert np.array_equal(np.nan_to_num(ev[0], nan=7.0), np.nan_to_num(ev[1], nan=7.0))


def test_integer_tree_and_forest_round_trip(gpu, tmp_path):
    from pptk_b200 import ragged
    kd = gpu.kdtree
    rng = np.random.default_rng(1)
    P = rng.integers(-30000, 30000, (20_000, 2)).astype(np.int16)
    t = kd._build(P)
    t.save(tmp_path / "i16.bin")
    u = kd.load(tmp_path / "i16.bin")
    assert u.dtype == np.int16
    assert np.array_equal(u.ref_nodes(), t.ref_nodes())
    for a, b in zip(kd.knn(u, None, 5), kd.knn(t, None, 5)):
        assert np.array_equal(a, b)
    sizes = rng.integers(0, 2000, 30)
    off = np.concatenate([[0], np.cumsum(sizes)])
    C = rng.random((off[-1], 3)).astype(np.float32)
    f = ragged.Forest(C, off)
    f.save(tmp_path / "forest.bin")
    g = ragged.Forest.load(tmp_path / "forest.bin", off)
    assert g.ncloud == f.ncloud and np.array_equal(g.valid_offsets, f.valid_offsets)
    for a, b in zip(g.knn(7), f.knn(7)):
        assert np.array_equal(a, b)
    assert np.array_equal(np.nan_to_num(g.normals(7)), np.nan_to_num(f.normals(7)))
    with pytest.raises(ValueError):
        ragged.Forest.load(tmp_path / "forest.bin", off[:-1])


def test_damaged_files_are_refused(gpu, tmp_path):
    kd = gpu.kdtree
    P = np.random.default_rng(2).random((5000, 3)).astype(np.float32)
    t = kd._build(P)
    t.save(tmp_path / "t.bin")
    good = bytearray((tmp_path / "t.bin").read_bytes())

    def refused(data, match):
        p = tmp_path / "bad.bin"
        p.write_bytes(bytes(data))
        with pytest.raises(ValueError, match=match):
            kd.load(p)

    flipped = bytearray(good)
    flipped[len(good) // 2] ^= 0x40
    refused(flipped, "checksum")
    refused(good[: len(good) - 100], "shorter")
    refused(b"NOTATREE" + bytes(good[8:]), "not a pptk_b200 tree")
    # a node reference far outside the node array, with a matching checksum:
    # the device check refuses it before any query can follow it
    sec = np.frombuffer(bytes(good[SECTIONS_AT:SECTIONS_AT + 64]), dtype="<i8")
    pad = [(int(b) + 63) // 64 * 64 for b in sec]
    tnodes_at = HEADER + pad[0] + pad[1] + pad[2]
    bad = bytearray(good)
    bad[tnodes_at + 48:tnodes_at + 52] = np.int32(1 << 28).tobytes()  # node 0, child 0 reference
    bad[tnodes_at + 56:tnodes_at + 60] = np.int32(5).tobytes()        # with a non-zero count
    bad[HASH_AT:HASH_AT + 8] = np.uint64(_fnv_words(bytes(bad[HEADER:]))).tobytes()
    refused(bad, "out of range")
    # the intact file still loads
    u = kd.load(tmp_path / "t.bin")
    assert np.array_equal(kd.knn(u, None, 4)[0], kd.knn(t, None, 4)[0])
