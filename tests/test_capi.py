"""The C-ABI library loads, exports every declared symbol, refuses malformed
inputs, and fails loudly without a GPU."""
import re
from pathlib import Path

import pytest

import parcomm_b200 as qf

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "parcomm_qafold.h").read_text()
    return sorted(set(re.findall(r"^(?:int|void|size_t|uint64_t)\s+(qf_\w+)\s*\(", text, re.M)))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    for n in ("qf_params_new", "qf_commit", "qf_prove", "qf_verify", "qf_eval_claims", "qf_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = qf.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing


def test_params_and_statement_without_gpu(vectors):
    p = qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=10, packed_log=4))
    g = vectors["f65521_demo"]
    assert (p.active, p.logical, p.blocks) == (g["active_entries"], g["logical_entries"], g["pcs_blocks"])
    import json
    st = json.loads(p.statement_json([bytes(range(i, i + 32)) for i in range(4)]))
    assert list(st) == ["version", "config", "shapes", "parameter_digest", "roots"]
    assert st["version"] == 2 and st["config"] == {"chunk_log": 10, "packed_log": 4, "query_rf_bits": 100}
    assert st["shapes"][0] == {"rows": 31, "cols": 37} and bytes(st["parameter_digest"]) == p.parameter_digest
    assert [bytes(r) for r in st["roots"]] == [bytes(range(i, i + 32)) for i in range(4)]


def test_invalid_config_rejected():
    with pytest.raises(qf.QfError, match="invalid ParComm config"):
        qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=9, packed_log=4))
    with pytest.raises(qf.QfError, match="invalid ParComm config"):
        qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=10, packed_log=7))
    with pytest.raises(qf.QfError, match="invalid matrix shape"):
        qf.Parameters([(0, 4)], qf.Config(chunk_log=10, packed_log=4))


def test_commit_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=10, packed_log=4))
    import numpy as np
    with pytest.raises(qf.QfError) as e:
        p.commit(np.zeros(p.active, dtype=np.int8))
    assert e.value.code == qf.QF_E_NO_DEVICE


def test_koalabear_params_and_recompute_mode_without_gpu(vectors):
    """The KoalaBear^4 parameter set mirrors the reference's layout facts, and
    every commit mode refuses to run without a device (no CPU fallback)."""
    import torch
    import numpy as np
    p = qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=10, packed_log=4), field=qf.FIELD_KOALABEAR)
    g = vectors["koalabear_demo"]
    assert (p.active, p.logical, p.blocks) == (g["active_entries"], g["logical_entries"], g["pcs_blocks"])
    assert p.weight_dtype == np.int16
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    for commit in (lambda: p.commit(np.zeros(p.active, dtype=np.int16)),
                   lambda: p.commit_recomputed(np.zeros(p.active, dtype=np.int16))):
        with pytest.raises(qf.QfError) as e:
            commit()
        assert e.value.code == qf.QF_E_NO_DEVICE


def test_wrong_weight_width_rejected():
    import torch
    p = qf.Parameters(qf.demo_shapes(), qf.Config(chunk_log=10, packed_log=4), field=qf.FIELD_KOALABEAR)
    with pytest.raises(qf.QfError, match="int16"):
        p.commit_recomputed(torch.zeros(p.active, dtype=torch.int8))


@pytest.mark.parametrize("field", [qf.FIELD_F65521, qf.FIELD_KOALABEAR])
def test_malformed_inputs_rejected(field):
    """end_to_end.rs:194-213: no matrices, a zero dimension and a dimension
    whose size overflows are refused; a BVA one value short and a claim with a
    missing coordinate are rejected."""
    import dataclasses
    import oracle
    from parcomm_b200 import layout
    cfg = qf.Config(chunk_log=10, packed_log=4)
    for shapes, msg in (([], "invalid matrix count"), ([(0, 1)], "invalid matrix shape"),
                        ([(2**64 - 1, 2)], "invalid matrix shape")):
        with pytest.raises(qf.QfError, match=msg):
            qf.Parameters(shapes, cfg, field=field)
    name = "f65521" if field == qf.FIELD_F65521 else "koalabear"
    shapes = [(3, 5)]
    import numpy as np
    bva = layout.encode(shapes, layout.demo_matrices(shapes, dtype=np.int8 if name == "f65521" else np.int16))
    with pytest.raises(oracle.OracleError, match="active BVA length"):
        oracle.prove(shapes, 10, 4, bva[:-1], field=name)
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva, field=name)
    p = qf.Parameters(shapes, cfg, field=field)
    c = qf.claims_from_bytes(p.shapes, claims)[0]
    with pytest.raises(qf.QfError):
        p.verify([roots], [dataclasses.replace(c, row=c.row[:-1])], proof)
    assert not oracle.verify(shapes, 10, 4, roots, claims[16:], proof, field=name)
    p.verify([roots], [c], proof)


@pytest.mark.parametrize("field", [qf.FIELD_F65521, qf.FIELD_KOALABEAR])
def test_library_points_and_claim_codec_match_the_oracle(field):
    """The library's benchmark points for a multi-block statement (main.rs:190-204)
    are the points of the oracle's claims, and the claim codec round-trips
    the oracle's claim bytes."""
    import numpy as np
    import oracle
    from parcomm_b200 import layout
    name = "f65521" if field == qf.FIELD_F65521 else "koalabear"
    shapes = [(31, 37), (65, 17), (1, 7), (9, 1), (300, 40)]
    dt = np.int8 if name == "f65521" else np.int16
    bva = layout.encode(shapes, layout.demo_matrices(shapes, dtype=dt))
    roots, claims, _, _ = oracle.prove(shapes, 10, 4, bva, field=name)
    p = qf.Parameters(shapes, qf.Config(chunk_log=10, packed_log=4), field=field)
    rs = [roots[i:i + 32] for i in range(0, len(roots), 32)]
    assert len(rs) == p.blocks > 1
    cl = qf.claims_from_bytes(p.shapes, claims)
    assert qf.claims_to_bytes(cl) == claims
    points = qf.claims_from_bytes(p.shapes, p.benchmark_points(rs), with_value=False)
    assert [(c.row, c.col) for c in points] == [(c.row, c.col) for c in cl]


def test_sharded_prove_checks_its_arguments_and_needs_a_device():
    """qf_prove_sharded refuses a rank outside [0, world) and, with valid
    arguments, fails loudly without a device (no CPU fallback)."""
    import numpy as np
    import torch
    p = qf.Parameters([(300, 700), (129, 65)], qf.Config(chunk_log=14, packed_log=4))
    v = np.zeros(p.active, dtype=np.int8)
    for rank, world in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(qf.QfError) as e:
            p.prove_sharded(v, rank, world, lambda b: b * max(world, 1))
        assert e.value.code == qf.QF_E_ARGUMENT
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(qf.QfError) as e:
        p.prove_sharded(v, 0, 2, lambda b: b * 2)
    assert e.value.code == qf.QF_E_NO_DEVICE
