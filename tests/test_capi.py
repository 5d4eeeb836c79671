"""The C-ABI library loads, exports every declared symbol, and fails loudly without a GPU."""
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
