"""Layout of the 8B-shape collection (226 matrices) and the smoke matrix."""
import parcomm_b200 as qf
from parcomm_b200 import layout


def shapes_8b():
    s = []
    for _ in range(32):
        s += [(4096, 4096), (1024, 4096), (1024, 4096), (4096, 4096), (14336, 4096), (14336, 4096), (4096, 14336)]
    return [(128256, 4096)] + s + [(128256, 4096)]


def test_8b_shape_layout():
    bs, active, logical = layout.buckets(shapes_8b())
    assert len(shapes_8b()) == 226
    assert sum(r * c for r, c in shapes_8b()) == 8_029_995_008
    assert (len(bs), active, logical) == (424, 8_053_063_680, 1 << 33)


def test_python_layout_matches_library():
    p = qf.Parameters(shapes_8b()[1:4] + [(31, 37)], qf.Config(chunk_log=20, packed_log=4))
    bs, active, logical = layout.buckets(p.shapes)
    assert (p.active, p.logical, p.buckets) == (active, logical, len(bs))


def test_intervals_last_doubled():
    assert layout.intervals(31) == [(0, 16), (16, 8), (24, 4), (28, 4)]
    assert layout.intervals(37) == [(0, 32), (32, 4), (36, 1)]
    assert layout.intervals(128256) == [(0, 65536), (65536, 32768), (98304, 16384), (114688, 16384)]


def test_layout_of_a_70b_scale_matrix_without_its_weights():
    """cpu_optimization.rs:33-40: a 2^18 x (2^18 + 16) matrix lays out to more
    than 2^36 active entries in 2^37 logical ones, 128 blocks of 2^30; a
    2^20 x 2^20 matrix exceeds the 2^37-entry capacity and is refused."""
    _, active, logical = layout.buckets([(1 << 18, (1 << 18) + 16)])
    assert active > 1 << 36 and logical == 1 << 37 and logical // (1 << 30) == 128
    p = qf.Parameters([(1 << 18, (1 << 18) + 16)], qf.Config(chunk_log=30, packed_log=4))
    assert (p.active, p.logical, p.blocks) == (active, logical, 128)
    import pytest
    with pytest.raises(qf.QfError, match="matrix exceeds supported capacity"):
        qf.Parameters([(1 << 20, 1 << 20)], qf.Config(chunk_log=30, packed_log=4))


def test_real_8b_layout_matches_the_reference_fixture(vectors):
    """end_to_end.rs:262-298: the reference's 291-tensor 8B layout fixture,
    bucket by bucket (matrix, offset, row and column offsets, lengths and
    physical lengths), through the table's BLAKE2s, and the counts, for the
    Python layout and the host C++ layout; the library agrees on the counts."""
    import hashlib
    import struct
    g = vectors["llama8b_layout"]
    shapes = [tuple(s) for s in g["shapes"]]
    bs, active, logical = layout.buckets(shapes)
    assert (len(shapes), len(bs), active, logical) == (291, g["bucket_count"], g["active_entries"], g["logical_entries"])
    h = hashlib.blake2s()
    for b in bs:
        h.update(struct.pack("<8Q", b.matrix, b.offset, b.row_offset, b.col_offset, b.rows, b.cols,
                             b.physical_rows, b.physical_cols))
    assert h.hexdigest() == g["buckets_blake2s"]
    import oracle
    rows, h_active, h_logical = oracle.host_layout(shapes)
    h = hashlib.blake2s()
    for r in rows:
        h.update(struct.pack("<8Q", *r))
    assert (h.hexdigest(), h_active, h_logical) == (g["buckets_blake2s"], active, logical)
    p = qf.Parameters(shapes, qf.Config(chunk_log=30, packed_log=4))
    assert (p.active, p.logical, p.buckets) == (active, logical, len(bs))
