"""The two entropy-decoder modes give the same codes.

`k_decode` decodes a plane with one warp (speculative slices, then
resynchronisation) or, for dense streams of at least 16384 planes in
launches of at least 128 work items, with one thread. The threshold on the
mean payload bits per plane is read once per process from
STZ_DECODE_SEQ_BITS, so each mode runs in a fresh process: 0 sends every
large stream of a large launch to the one-thread decoder, 4294967295 keeps
every plane on the warp decoder. On the 512^3 lognormal stream (finest
streams: 16384 planes each) both must give the default decode's output bit
for bit; the default decode itself is pinned to the oracle's in
test_gpu_configs."""
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import hashlib, sys
sys.path[:0] = [sys.argv[1]]
import numpy as np, torch
import stz_b200
from stz_b200 import fields
ctx = stz_b200.Context(0)
f = fields.lognormal((512, 512, 512), 2025, np.float32, device="cuda:0")
s = ctx.compress(f, eb=1e-3, eb_mode="rel")
out = torch.empty_like(f)
ctx.decompress(s, out=out)
print(hashlib.sha256(out.view(torch.int32).cpu().numpy().tobytes()).hexdigest())
"""


def _child_hash(seq_bits):
    env = dict(os.environ, STZ_DECODE_SEQ_BITS=str(seq_bits))
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "sc25-stz2_b200")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip().splitlines()[-1]


def test_sequential_and_warp_decoders_agree(ctx):
    from stz_b200 import fields

    f = fields.lognormal((512, 512, 512), 2025, np.float32, device="cuda:0")
    s = ctx.compress(f, eb=1e-3, eb_mode="rel")
    out = torch.empty_like(f)
    ctx.decompress(s, out=out)
    want = hashlib.sha256(out.view(torch.int32).cpu().numpy().tobytes()).hexdigest()
    del f, out, s
    torch.cuda.empty_cache()
    assert _child_hash(0) == want
    assert _child_hash(4294967295) == want
