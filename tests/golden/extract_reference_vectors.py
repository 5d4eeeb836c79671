"""Regenerates reference_vectors.json from the reference's own files (read as text).

Run in the development container where the reference checkout is mounted:
    python tests/golden/extract_reference_vectors.py /path/to/reference
Sources:
  * validation/qafold8-smoke-final/run.log  (F65521 demo bundle: proof bytes,
    proof BLAKE2s printed with `{:x?}` (no zero padding), commitment JSON size)
  * validation/qafold16-smoke/run.log       (KoalaBear demo bundle)
  * qafold/f65521/vendor/qafold/src/qafold_short_pc.rs  (native opening +
    Decide wire fixture digest, test `native_opening_and_decide_wire_fixture`)
  * qafold/f65521/tests/fixtures/llama8b-layout.json  (the real 8B layout of
    end_to_end.rs:262-298: its 291 shapes, the counts, and a BLAKE2s of the
    bucket table, eight little-endian u64 per bucket in layout order)
"""
import json
import re
import sys
from pathlib import Path


def smoke(path: Path) -> dict:
    for line in path.read_text().splitlines():
        if '"proof_blake2s"' in line:
            rec = json.loads(line)
            digest = "".join(f"{int(x, 16):02x}" for x in rec["proof_blake2s"].strip("[]").split(", "))
            return {"proof_bytes": rec["proof_bytes"], "proof_blake2s": digest,
                    "public_commitment_json_bytes": rec["public_commitment_json_bytes"],
                    "active_entries": rec["active_entries"], "logical_entries": rec["logical_entries"],
                    "bucket_count": rec["bucket_count"], "pcs_blocks": rec.get("verifier_profile", {}).get("authenticated_roots"),
                    "source": str(path.relative_to(path.parents[2]))}
    raise SystemExit(f"no proof record in {path}")


def wire_fixture(path: Path) -> dict:
    text = path.read_text()
    i = text.index("fn native_opening_and_decide_wire_fixture")
    block = text[i:]
    arr = re.search(r"assert_eq!\(\s*digest,\s*\[(.*?)\]", block, re.S).group(1)
    digest = "".join(f"{int(x, 16):02x}" for x in re.findall(r"0x([0-9a-fA-F]{2})", arr))
    line = text[:i].count("\n") + 1
    return {"blake2s_root_opening_decide": digest, "source": f"qafold/f65521/vendor/qafold/src/qafold_short_pc.rs:{line}",
            "pcs": {"n_witness": 65536, "extension_columns": 16, "index": 2, "security_bits": 80},
            "rng_seed_u64": "0x706172616c6c656c"}


BUCKET_FIELDS = ("tensor_index", "dense_offset", "row_offset", "col_offset", "row_len", "col_len",
                 "physical_row_len", "physical_col_len")


def bucket_table_digest(rows) -> str:
    """BLAKE2s-256 of the bucket table: per bucket the eight fields above as u64 LE."""
    import hashlib
    import struct
    h = hashlib.blake2s()
    for r in rows:
        h.update(struct.pack("<8Q", *r))
    return h.hexdigest()


def layout_fixture(path: Path) -> dict:
    fx = json.loads(path.read_text())
    rows = [[b[k] for k in BUCKET_FIELDS] for b in fx["buckets"]]
    return {"shapes": fx["shapes"], "bucket_count": len(rows), "active_entries": fx["layout"]["active_entries"],
            "logical_entries": fx["layout"]["logical_entries"], "buckets_blake2s": bucket_table_digest(rows),
            "source": "qafold/f65521/tests/fixtures/llama8b-layout.json"}


def main(ref: Path) -> None:
    out = {
        "f65521_demo": smoke(ref / "validation/qafold8-smoke-final/run.log"),
        "koalabear_demo": smoke(ref / "validation/qafold16-smoke/run.log"),
        "f65521_wire_fixture": wire_fixture(ref / "qafold/f65521/vendor/qafold/src/qafold_short_pc.rs"),
        "demo_command": "demo --chunk-log 10 --packed-log 4 --cache-mode recompute",
        "llama8b_layout": layout_fixture(ref / "qafold/f65521/tests/fixtures/llama8b-layout.json"),
    }
    dst = Path(__file__).with_name("reference_vectors.json")
    dst.write_text(json.dumps(out, indent=2) + "\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: extract_reference_vectors.py <reference checkout>")
    main(Path(sys.argv[1]))
