"""The reference's dense BVA stream format on the CPU: the description a
converter writes, exact-length reads (short and excess input rejected), the
format, dtype and layout checks with the reference's messages, and int16
payloads little-endian (qafold/f65521/src/main.rs:116-173,
qafold/koalabear/src/main.rs:116-177, tests/cli_stream.py)."""
import io
import json

import numpy as np
import pytest

import parcomm_b200 as qf
from parcomm_b200 import layout, stream


def cli_stream_case():
    # The description and data of the reference's CLI stream test (cli_stream.py:11-16).
    d = {"format": "parcomm-dense-bva-stream-description", "storage_dtype": "i8",
         "shapes": [[32, 32]], "stream_bytes": 1024, "layout": {"logical_entries": 1024}}
    return d, bytes((i * 73) % 256 for i in range(1024))


def test_describe_matches_the_reference_description():
    d, _ = cli_stream_case()
    assert stream.describe([(32, 32)]) == d
    assert json.loads(json.dumps(stream.describe([(31, 37), (9, 1)], "i16")))["storage_dtype"] == "i16"


def test_read_the_reference_case():
    d, data = cli_stream_case()
    m = stream.open_stream(d, io.BytesIO(data), qf.Config(10, 4), pinned=False)
    assert m.params.shapes == [qf.Shape(32, 32)] and m.params.active == 1024
    assert np.array_equal(m.bva, np.frombuffer(data, dtype=np.int8))


@pytest.mark.parametrize("tail", [-1, 1])
def test_short_and_excess_input_are_rejected(tail):
    d, data = cli_stream_case()
    src = data[:-1] if tail < 0 else data + b"\0"
    with pytest.raises(qf.QfError, match="truncated BVA input" if tail < 0 else "excess BVA input"):
        stream.open_stream(d, io.BytesIO(src), qf.Config(10, 4), pinned=False)


def test_foreign_format_dtype_and_layout_are_rejected():
    d, data = cli_stream_case()
    for key, value, msg in [("format", "other", "requires signed-i8"), ("stream_bytes", 1023, "layout mismatch"),
                            ("layout", {"logical_entries": 2048}, "layout mismatch"),
                            ("shapes", [[32, 33]], "layout mismatch")]:
        bad = dict(d, **{key: value})
        with pytest.raises(qf.QfError, match=msg):
            stream.read_description(bad)
    # Each reference binary takes only its own dtype.
    with pytest.raises(qf.QfError, match="requires signed-i16"):
        stream.read_description(d, storage_dtype="i16")


def test_int16_payloads_round_trip_little_endian(tmp_path):
    shapes = [(31, 37), (65, 17), (1, 7), (9, 1)]
    rng = np.random.default_rng(4)
    mats = [rng.integers(-32768, 32768, size=s).astype(np.int16) for s in shapes]
    bva = layout.encode(shapes, mats, np.int16)
    bva[0] = 0x0102
    desc, raw = tmp_path / "input.json", tmp_path / "input.bva"
    d = stream.write_stream(desc, raw, shapes, bva)
    assert d["storage_dtype"] == "i16" and d["stream_bytes"] == 2 * bva.size
    assert raw.read_bytes()[:2] == b"\x02\x01"
    m = stream.open_stream(desc, raw, qf.Config(10, 4), pinned=False)
    assert m.params.field == qf.FIELD_KOALABEAR and np.array_equal(m.bva, bva)


def test_reads_span_several_pieces(tmp_path, monkeypatch):
    monkeypatch.setattr(stream, "_PIECE", 1000)
    shapes = [(300, 700), (129, 65)]
    rng = np.random.default_rng(5)
    bva = layout.encode(shapes, [rng.integers(-128, 128, size=s).astype(np.int8) for s in shapes], np.int8)
    stream.write_stream(tmp_path / "d.json", tmp_path / "s.bva", shapes, bva)
    m = stream.open_stream(tmp_path / "d.json", tmp_path / "s.bva", qf.Config(14, 4), pinned=False)
    assert np.array_equal(m.bva, bva)


def test_reads_stdin_like_the_reference_cli(tmp_path):
    """`--input -` (main.rs:155-157): the stream comes on standard input."""
    import subprocess
    import sys
    from pathlib import Path
    d, data = cli_stream_case()
    (tmp_path / "input.json").write_text(json.dumps(d))
    code = ("import sys; import parcomm_b200 as qf; from parcomm_b200 import stream; "
            "m = stream.open_stream(sys.argv[1], '-', qf.Config(10, 4), pinned=False); "
            "sys.stdout.write(m.bva.tobytes().hex())")
    root = Path(__file__).resolve().parents[1]
    ok = subprocess.run([sys.executable, "-c", code, str(tmp_path / "input.json")], input=data, capture_output=True,
                        cwd=root, timeout=120)
    assert ok.returncode == 0, ok.stderr.decode()
    assert bytes.fromhex(ok.stdout.decode()) == data
    extra = subprocess.run([sys.executable, "-c", code, str(tmp_path / "input.json")], input=data + b"\0",
                           capture_output=True, cwd=root, timeout=120)
    assert extra.returncode != 0 and b"excess BVA input" in extra.stderr
