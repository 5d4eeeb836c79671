"""The oracle's OpenMP loops (lane projections, EO and sumcheck rounds,
Mobius levels, factor and equality tables) give the same proof bytes with
one thread as with several: field sums do not depend on their order.  Runs
on the CPU in two fresh processes."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

CODE = r"""
import hashlib, json, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {oracle!r})
import oracle
from parcomm_b200 import layout
shapes = [(1024, 4096), (300, 700), (1, 5000)]
rng = np.random.default_rng(5)
mats = [np.clip(np.rint(rng.normal(0, 20, r * c)), -127, 127).astype(np.int8).reshape(r, c) for r, c in shapes]
bva = layout.encode(shapes, mats)
roots, claims, proof, _ = oracle.prove(shapes, 20, 4, bva)
print(json.dumps([hashlib.blake2s(b).hexdigest() for b in (roots, claims, proof)]))
"""


def run(threads: int):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([sys.executable, "-c", CODE.format(root=str(ROOT), oracle=str(ROOT / "oracle"))], env=env,
                         capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_oracle_bytes_do_not_depend_on_the_thread_count():
    assert run(1) == run(4)
