"""Launch chaining inside a solve (programmatic dependent launch) changes when a
kernel's blocks start, never what they compute: the same solve with the chaining
on (default) and off (DECO_PDL=0, read once per process) must give bit-identical
solutions and the same iteration counts, in float64 and in mixed precision.  A
kernel that read its predecessor's output before its dependency wait would make
the two differ."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import hashlib, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import deco_b200 as d
from deco_b200 import gen
from conftest import cpr_json, sol_json
out = {}
for bits in (64, 32):
    s = gen.grid(40, 30, 20, bs=2, seed=5)
    A = d.CSR.from_system(s)
    b = torch.from_numpy(s.b.copy()).cuda()
    P = d.CPR(cpr_json(2), A, b, precision=bits)
    S = d.SOL(sol_json(), A, P, b, precision=bits)
    x = S.x.cpu().numpy()
    out[str(bits)] = {"iter": S.iter, "flag": S.flag, "sha": hashlib.sha256(x.tobytes()).hexdigest()}
print(json.dumps(out))
"""


def run_child(pdl):
    # the autotuner's timing could pick another product layout in one process than in
    # the other; the layout rules alone keep the two runs' arithmetic the same
    env = dict(os.environ, DECO_PDL=pdl, DECO_AUTOTUNE="0")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT], cwd=os.path.join(ROOT, "tests"), env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_chained_launches_give_identical_solves():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    on, off = run_child("1"), run_child("0")
    for bits in ("64", "32"):
        assert on[bits]["flag"] == 0 and off[bits]["flag"] == 0
        assert on[bits]["iter"] == off[bits]["iter"], (bits, on[bits], off[bits])
        assert on[bits]["sha"] == off[bits]["sha"], f"precision {bits}: the solutions differ bit-wise"
