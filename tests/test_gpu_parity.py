"""GPU proofs are byte-identical to the CPU oracle's (and to the reference's
golden demo digest), through the C ABI.  Requires a B200."""
import hashlib

import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

pytestmark = pytest.mark.gpu


def blake2s(b: bytes) -> str:
    return hashlib.blake2s(b, digest_size=32).hexdigest()


def gaussian_i8(rng, n, sigma=20.0, forced=0.0):
    v = np.clip(np.rint(rng.normal(0.0, sigma, n)), -127, 127).astype(np.int8)
    if forced:
        idx = rng.choice(n, max(1, int(n * forced)), replace=False)
        v[idx] = np.where(rng.random(idx.size) < 0.5, -127, 127).astype(np.int8)
    return v


def gaussian_i16(rng, n, sigma=3000.0, forced=0.0):
    v = np.clip(np.rint(rng.normal(0.0, sigma, n)), -32768, 32767).astype(np.int16)
    if forced:
        idx = rng.choice(n, max(1, int(n * forced)), replace=False)
        v[idx] = np.where(rng.random(idx.size) < 0.5, -32768, 32767).astype(np.int16)
    return v


FIELDS = {"f65521": qf.FIELD_F65521, "koalabear": qf.FIELD_KOALABEAR}


def run_both(shapes, chunk_log, packed_log, mats, field="f65521"):
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=packed_log), field=FIELDS[field])
    bva = layout.encode(p.shapes, mats)
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, packed_log, bva, field=field)
    c = p.commit(bva)
    assert b"".join(c.roots) == o_roots, "commitment roots differ"
    claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
    assert qf.claims_to_bytes(claims) == o_claims, "claims differ"
    proof, prof = p.prove(c, claims)
    assert proof.to_bytes() == o_proof, "proof bytes differ"
    p.verify(c.roots, claims, proof)
    assert oracle.verify(p.shapes, chunk_log, packed_log, o_roots, o_claims, proof.to_bytes(), field=field)
    c.close()
    return proof, prof


def test_demo_bundle_matches_reference_digest(vectors):
    shapes = qf.demo_shapes()
    proof, prof = run_both(shapes, 10, 4, layout.demo_matrices(shapes))
    assert len(proof.to_bytes()) == vectors["f65521_demo"]["proof_bytes"]
    assert blake2s(proof.to_bytes()) == vectors["f65521_demo"]["proof_blake2s"]
    assert prof.kernel_launches > 0


def test_smoke_config_1024x4096_chunk20():
    rng = np.random.default_rng(0)
    mats = [gaussian_i8(rng, 1024 * 4096).reshape(1024, 4096)]
    run_both([(1024, 4096)], 20, 4, mats)


@pytest.mark.parametrize("packed_log", [1, 4, 6])
def test_ragged_shapes_multilevel(packed_log):
    rng = np.random.default_rng(7 + packed_log)
    shapes = [(300, 700), (129, 65), (1, 5000), (77, 1)]
    mats = [gaussian_i8(rng, r * c, forced=0.001).reshape(r, c) for r, c in shapes]
    run_both(shapes, 14, packed_log, mats)


@pytest.mark.parametrize("rows,chunk_log", [(4096, 24), (2048, 23), (4096, 25)])
def test_single_matrix_deep_code_sequences(rows, chunk_log):
    """One matrix per statement, as in the per-matrix path: chunk 23-25 give
    code sequences whose Decide levels with a carried codeword have 2^10 to
    2^12 rows, run on the device."""
    rng = np.random.default_rng(rows + chunk_log)
    mats = [gaussian_i8(rng, rows * 4096, forced=0.001).reshape(rows, 4096)]
    run_both([(rows, 4096)], chunk_log, 4, mats)


def test_single_block_opening():
    rng = np.random.default_rng(3)
    mats = [gaussian_i8(rng, 64 * 64).reshape(64, 64)]
    run_both([(64, 64)], 12, 4, mats)


def test_zero_suffix_blocks_share_one_commitment():
    rng = np.random.default_rng(5)
    shapes = [(1024, 1024), (1, 16)]
    mats = [gaussian_i8(rng, r * c).reshape(r, c) for r, c in shapes]
    proof, _ = run_both(shapes, 16, 4, mats)


def test_extreme_values_and_all_zero():
    shapes = [(256, 256), (3, 3)]
    mats = [np.full((256, 256), -127, np.int8), np.zeros((3, 3), np.int8)]
    mats[0][::7, ::3] = 127
    run_both(shapes, 12, 3, mats)


def test_nonzero_padding_rejected():
    p = qf.Parameters([(31, 31)], qf.Config(chunk_log=10, packed_log=4))
    bva = layout.encode(p.shapes, [np.ones((31, 31), np.int8)])
    bs, _, _ = layout.buckets(p.shapes)
    b = next(b for b in bs if b.cols > b.physical_cols)
    bva[b.offset + b.physical_cols] = 1
    with pytest.raises(qf.QfError, match="nonzero boundary padding"):
        p.commit(bva)


# ---------------------------------------------------------------- KoalaBear^4, signed 16-bit payloads
def test_koalabear_demo_bundle_matches_reference_digest(vectors):
    shapes = qf.demo_shapes()
    proof, prof = run_both(shapes, 10, 4, layout.demo_matrices(shapes, dtype=np.int16), field="koalabear")
    assert len(proof.to_bytes()) == vectors["koalabear_demo"]["proof_bytes"]
    assert blake2s(proof.to_bytes()) == vectors["koalabear_demo"]["proof_blake2s"]
    assert prof.kernel_launches > 0


@pytest.mark.parametrize("packed_log", [1, 4, 6])
def test_koalabear_ragged_shapes_multilevel(packed_log):
    rng = np.random.default_rng(70 + packed_log)
    shapes = [(300, 700), (129, 65), (1, 5000), (77, 1)]
    mats = [gaussian_i16(rng, r * c, forced=0.001).reshape(r, c) for r, c in shapes]
    run_both(shapes, 14, packed_log, mats, field="koalabear")


def test_koalabear_1024x4096_chunk20():
    rng = np.random.default_rng(11)
    mats = [gaussian_i16(rng, 1024 * 4096).reshape(1024, 4096)]
    run_both([(1024, 4096)], 20, 4, mats, field="koalabear")


@pytest.mark.parametrize("rows,chunk_log", [(2048, 23), (4096, 24)])
def test_koalabear_single_matrix_deep_code_sequences(rows, chunk_log):
    rng = np.random.default_rng(rows + chunk_log + 1)
    mats = [gaussian_i16(rng, rows * 4096, forced=0.001).reshape(rows, 4096)]
    run_both([(rows, 4096)], chunk_log, 4, mats, field="koalabear")


def test_koalabear_single_block_and_zero_suffix():
    rng = np.random.default_rng(13)
    run_both([(64, 64)], 12, 4, [gaussian_i16(rng, 64 * 64).reshape(64, 64)], field="koalabear")
    shapes = [(1024, 1024), (1, 16)]
    mats = [gaussian_i16(rng, r * c).reshape(r, c) for r, c in shapes]
    run_both(shapes, 16, 4, mats, field="koalabear")


def test_koalabear_extreme_values_and_all_zero():
    shapes = [(256, 256), (3, 3)]
    mats = [np.full((256, 256), -32768, np.int16), np.zeros((3, 3), np.int16)]
    mats[0][::7, ::3] = 32767
    run_both(shapes, 12, 3, mats, field="koalabear")


def test_koalabear_nonzero_padding_rejected():
    p = qf.Parameters([(31, 31)], qf.Config(chunk_log=10, packed_log=4), field=qf.FIELD_KOALABEAR)
    bva = layout.encode(p.shapes, [np.ones((31, 31), np.int16)])
    bs, _, _ = layout.buckets(p.shapes)
    b = next(b for b in bs if b.cols > b.physical_cols)
    bva[b.offset + b.physical_cols] = 1
    with pytest.raises(qf.QfError, match="nonzero boundary padding"):
        p.commit(bva)


# ---------------------------------------------------------------- recompute mode over streamed host weights
def run_streamed(shapes, chunk_log, packed_log, mats, field="f65521", resident_bytes=0, pinned=False):
    """commit_recomputed: the weights stay in host memory and every pass
    streams them block by block; the bytes must equal the oracle's."""
    import torch
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=packed_log), field=FIELDS[field])
    bva = layout.encode(p.shapes, mats)
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, packed_log, bva, field=field)
    host = torch.from_numpy(bva).pin_memory() if pinned else bva
    c = p.commit_recomputed(host, resident_bytes=resident_bytes)
    h2d, resident, live = c.stream_info()
    assert h2d == bva.nbytes and live == -(-bva.size // (1 << chunk_log))
    if resident_bytes is None:
        assert resident == live
    assert b"".join(c.roots) == o_roots, "commitment roots differ"
    claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
    assert qf.claims_to_bytes(claims) == o_claims, "claims differ"
    proof, _ = p.prove(c, claims)
    assert proof.to_bytes() == o_proof, "proof bytes differ"
    p.verify(c.roots, claims, proof)
    c.close()
    return proof


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_streamed_demo_bundle_matches_reference_digest(vectors, field):
    shapes = qf.demo_shapes()
    dt = np.int16 if field == "koalabear" else np.int8
    proof = run_streamed(shapes, 10, 4, layout.demo_matrices(shapes, dtype=dt), field=field)
    assert blake2s(proof.to_bytes()) == vectors[f"{field}_demo"]["proof_blake2s"]


@pytest.mark.parametrize("field,packed_log,resident,pinned", [
    ("f65521", 4, 0, True), ("f65521", 6, 3, False), ("koalabear", 4, 0, False), ("koalabear", 6, 2, True)])
def test_streamed_ragged_shapes_many_blocks(field, packed_log, resident, pinned):
    rng = np.random.default_rng(100 + packed_log + resident)
    shapes = [(300, 700), (129, 65), (1, 5000), (77, 1)]
    gen = gaussian_i16 if field == "koalabear" else gaussian_i8
    mats = [gen(rng, r * c, forced=0.001).reshape(r, c) for r, c in shapes]
    w = 2 if field == "koalabear" else 1
    run_streamed(shapes, 14, packed_log, mats, field=field, resident_bytes=resident * (1 << 14) * w, pinned=pinned)


@pytest.mark.parametrize("field,resident", [("f65521", 0), ("koalabear", None)])
def test_streamed_terms_spanning_blocks_and_zero_suffix(field, resident):
    """A 2^20-entry bucket spans 16 blocks of 2^16; 15 of 32 blocks are the
    zero suffix.  resident None: the automatic budget keeps every block."""
    rng = np.random.default_rng(17)
    shapes = [(1024, 1024), (1, 16)]
    gen = gaussian_i16 if field == "koalabear" else gaussian_i8
    mats = [gen(rng, r * c).reshape(r, c) for r, c in shapes]
    run_streamed(shapes, 16, 4, mats, field=field, resident_bytes=resident, pinned=True)


def test_streamed_matches_resident_commit_smoke_config():
    rng = np.random.default_rng(0)
    mats = [gaussian_i8(rng, 1024 * 4096).reshape(1024, 4096)]
    p = qf.Parameters([(1024, 4096)], qf.Config(chunk_log=20, packed_log=4))
    bva = layout.encode(p.shapes, mats)
    a = p.commit(bva)
    b = p.commit_recomputed(bva, resident_bytes=1 << 20)
    assert a.roots == b.roots
    claims = p.evaluate_claims(a, p.benchmark_points(a.roots))
    assert qf.claims_to_bytes(p.evaluate_claims(b, p.benchmark_points(b.roots))) == qf.claims_to_bytes(claims)
    pa, _ = p.prove(a, claims)
    pb, _ = p.prove(b, claims)
    assert pa.to_bytes() == pb.to_bytes()


def test_streamed_nonzero_padding_rejected():
    p = qf.Parameters([(31, 31), (40, 40)], qf.Config(chunk_log=10, packed_log=4))
    bva = layout.encode(p.shapes, [np.ones((31, 31), np.int8), np.ones((40, 40), np.int8)])
    bs, _, _ = layout.buckets(p.shapes)
    b = next(b for b in bs if b.cols > b.physical_cols)
    bva[b.offset + b.physical_cols] = 1
    with pytest.raises(qf.QfError, match="nonzero boundary padding"):
        p.commit_recomputed(bva)


@pytest.mark.parametrize("field,shapes,chunk_log", [
    ("f65521", [(300, 700), (129, 65), (1, 5000), (77, 1)], 14),   # many blocks
    ("koalabear", [(512, 1024)], 20),                              # one block
    ("f65521", [(64, 64)], 12)])                                   # one block
def test_recompute_mode_device_and_host_weights(field, shapes, chunk_log):
    """commit_recomputed over device-resident weights (read in place) and over
    host weights; single-block statements re-encode their block for the
    opening.  Both equal the oracle's bytes."""
    import torch
    rng = np.random.default_rng(23 + chunk_log)
    gen = gaussian_i16 if field == "koalabear" else gaussian_i8
    mats = [gen(rng, r * c, forced=0.001).reshape(r, c) for r, c in shapes]
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=4), field=FIELDS[field])
    bva = layout.encode(p.shapes, mats)
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, 4, bva, field=field)
    for weights in (torch.from_numpy(bva).cuda(), bva):
        c = p.commit_recomputed(weights)
        assert b"".join(c.roots) == o_roots
        claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
        assert qf.claims_to_bytes(claims) == o_claims
        proof, _ = p.prove(c, claims)
        assert proof.to_bytes() == o_proof
        c.close()


@pytest.mark.parametrize("mode", ["cache", "recompute_device", "recompute_host"])
def test_open_keeps_the_commitment_for_repeated_claims(mode):
    """qf_open answers several claims on one commitment; each proof equals the
    oracle's proof for those claims (fresh points per opening)."""
    import torch
    rng = np.random.default_rng(31)
    shapes = [(300, 700), (129, 65)]
    chunk_log = 14 if mode != "cache" else 16
    mats = [gaussian_i8(rng, r * c).reshape(r, c) for r, c in shapes]
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=4))
    bva = layout.encode(p.shapes, mats)
    if mode == "cache":
        c = p.commit(bva)
    elif mode == "recompute_device":
        c = p.commit_recomputed(torch.from_numpy(bva).cuda())
    else:
        c = p.commit_recomputed(bva)
    for k in range(3):
        n_coords = len(p.benchmark_points(c.roots)) // 16
        pts = rng.integers(0, 65521, n_coords * 8).astype("<u2").tobytes()  # canonical F65521^8 coordinates
        claims = p.evaluate_claims(c, pts)
        proof, _ = p.open(c, claims)
        _, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, 4, bva, claims=qf.claims_to_bytes(claims))
        assert qf.claims_to_bytes(claims) == o_claims
        assert proof.to_bytes() == o_proof, f"opening {k} differs"
        p.verify(c.roots, claims, proof)
    c.close()


def test_device_weights_written_just_before_commit():
    """Weights produced by torch kernels still in flight: the commit must see
    the finished tensor (the mirror synchronises the producer stream)."""
    import torch
    p = qf.Parameters([(4096, 4096)], qf.Config(chunk_log=22, packed_log=4))
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    roots = []
    for mode in ("cache", "recompute"):
        w = torch.randint(-127, 128, (4096 * 4096,), generator=g, device="cuda", dtype=torch.int32)
        w = (w * 3 + 1).clamp_(-127, 127).to(torch.int8)  # more work queued on torch's stream
        c = p.commit(w, on_device=True) if mode == "cache" else p.commit_recomputed(w)
        ref = p.commit(w.cpu().numpy())
        assert c.roots == ref.roots, mode
        roots.append(c.roots)
        c.close()
        ref.close()


@pytest.mark.parametrize("field,shapes,chunk_log,packed_log", [
    ("f65521", [(1, 70000), (70000, 1), (1, 1)], 16, 4),       # one row, one column, one entry
    ("koalabear", [(1, 70000), (3, 3)], 16, 1),
    ("koalabear", [(257, 513), (2, 65537)], 17, 6),
    ("f65521", [(1025, 1023)], 15, 2)])
def test_edge_shapes_every_mode(field, shapes, chunk_log, packed_log):
    """Thin and tiny shapes (buckets of one row or column, ragged padding on
    both axes) in cache mode and in recompute mode over device and host
    weights: the same bytes as the oracle."""
    import torch
    rng = np.random.default_rng(chunk_log * 10 + packed_log)
    gen = gaussian_i16 if field == "koalabear" else gaussian_i8
    mats = [gen(rng, r * c, forced=0.01).reshape(r, c) for r, c in shapes]
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=packed_log), field=FIELDS[field])
    bva = layout.encode(p.shapes, mats)
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, packed_log, bva, field=field)
    for mode in ("cache", "device", "host"):
        c = (p.commit(bva) if mode == "cache" else
             p.commit_recomputed(torch.from_numpy(bva).cuda() if mode == "device" else bva))
        assert b"".join(c.roots) == o_roots, mode
        claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
        assert qf.claims_to_bytes(claims) == o_claims, mode
        proof, _ = p.prove(c, claims)
        assert proof.to_bytes() == o_proof, mode
        c.close()


def test_all_zero_weights_streamed():
    shapes = [(512, 512), (100, 3)]
    p = qf.Parameters(shapes, qf.Config(chunk_log=14, packed_log=4), field=qf.FIELD_KOALABEAR)
    bva = layout.encode(p.shapes, [np.zeros(s, np.int16) for s in shapes])
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, 14, 4, bva, field="koalabear")
    c = p.commit_recomputed(bva)
    assert b"".join(c.roots) == o_roots
    claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
    proof, _ = p.prove(c, claims)
    assert proof.to_bytes() == o_proof


def test_greedy_pass_plan_runs_the_depth8_stage():
    """QF_TUNE=0 (the greedy split, read before the tuner's first use, hence a
    fresh process): the 8 Möbius levels above the tile of a chunk-23 statement
    run as one depth-8 strided pass, whose radix-4 stage on tile bits 4..5
    takes its groups in swapped order.  Roots and proof equal the oracle's."""
    import os
    import subprocess
    import sys
    import textwrap
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    code = textwrap.dedent("""
        import sys
        sys.path.insert(0, "oracle")
        import numpy as np
        import oracle
        import parcomm_b200 as qf
        from parcomm_b200 import layout
        rng = np.random.default_rng(123)
        w = np.clip(np.rint(rng.normal(0, 20, size=(2048, 4096))), -127, 127).astype(np.int8)
        p = qf.Parameters([(2048, 4096)], qf.Config(23, 4))
        bva = layout.encode(p.shapes, [w])
        o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, 23, 4, bva)
        c = p.commit(bva)
        assert b"".join(c.roots) == o_roots, "roots differ"
        claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
        assert qf.claims_to_bytes(claims) == o_claims, "claims differ"
        proof, _ = p.prove(c, claims)
        assert proof.to_bytes() == o_proof, "proof differs"
        print("greedy-ok")
    """)
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=dict(os.environ, QF_TUNE="0"),
                       capture_output=True, timeout=900)
    assert r.returncode == 0 and b"greedy-ok" in r.stdout, r.stderr.decode()[-3000:]


def test_device_setup_levels_chunk26():
    """Chunk 26 is the smallest block whose top setup level (2^14 encoded rows
    x 64 columns) is encoded and hashed on the device; the proof, which
    absorbs the parameter digest, equals the oracle's host-built one."""
    rng = np.random.default_rng(26)
    mats = [gaussian_i8(rng, 8192 * 8192, forced=0.001).reshape(8192, 8192)]
    run_both([(8192, 8192)], 26, 4, mats)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("chunk_log", [26, 28, 30])
def test_device_setup_digest_equals_host_setup(field, chunk_log):
    """The parameter digest of a device-built setup equals the one a process
    without a visible device builds on the host; the device setup also runs
    as a fresh process's first device work."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    shapes = [(1 << 15, 1 << 15)]
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=4), field=FIELDS[field])
    code = ("import parcomm_b200 as qf; "
            f"p = qf.Parameters({shapes!r}, qf.Config(chunk_log={chunk_log}, packed_log=4), field={FIELDS[field]!r}); "
            "print(p.parameter_digest.hex())")
    root = str(Path(__file__).resolve().parents[1])
    for visible in ("", None):
        env = dict(os.environ)
        if visible is not None:
            env["CUDA_VISIBLE_DEVICES"] = visible
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600, cwd=root)
        assert out.returncode == 0, out.stderr[-2000:]
        assert out.stdout.strip() == p.parameter_digest.hex()
