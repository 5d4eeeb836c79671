"""Every kernel choice writes the same bytes: the extension-product sums per
kernel as measured fastest (default), all on the CUDA cores and all on the
tensor cores (core_dots 1, 2), the tensor-core
weight passes (imma, F65521) and the per-matrix launch sequence, each
compared with the CPU oracle's proof.  Requires a B200."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

from test_gpu_parity import FIELDS, gaussian_i8, gaussian_i16

pytestmark = pytest.mark.gpu

OPTIONS = [{}, {"core_dots": 1}, {"core_dots": 2}, {"imma": 1}, {"per_matrix": 1}, {"core_dots": 2, "per_matrix": 1}]


def prove_with(p, bva, options):
    for k, v in options.items():
        qf.kernel_option(k, v)
    try:
        c = p.commit(bva)
        claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
        proof, _ = p.prove(c, claims)
        p.verify(c.roots, claims, proof)
        out = (b"".join(c.roots), qf.claims_to_bytes(claims), proof.to_bytes())
        c.close()
        return out
    finally:
        for k in options:
            qf.kernel_option(k, 0)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("chunk_log", [14, 20])
def test_kernel_options_write_oracle_bytes(field, chunk_log):
    rng = np.random.default_rng(chunk_log)
    shapes = [(300, 700), (129, 65), (1, 5000), (2048, 1024)] if chunk_log == 20 else [(300, 700), (129, 65), (1, 5000)]
    gen = gaussian_i16 if field == "koalabear" else gaussian_i8
    mats = [gen(rng, r * c, forced=0.001).reshape(r, c) for r, c in shapes]
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=4), field=FIELDS[field])
    bva = layout.encode(p.shapes, mats)
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, chunk_log, 4, bva, field=field)
    for options in OPTIONS:
        roots, claims, proof = prove_with(p, bva, options)
        assert roots == o_roots, f"roots differ with {options}"
        assert claims == o_claims, f"claims differ with {options}"
        assert proof == o_proof, f"proof bytes differ with {options}"


def test_unknown_kernel_option_is_an_error():
    with pytest.raises(qf.QfError):
        qf.kernel_option("no_such_option", 1)
    with pytest.raises(qf.QfError):
        qf.kernel_option("core_dots", 3)
