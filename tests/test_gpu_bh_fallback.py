"""The batched Barnes-Hut walk (FX_BH_FAST) starts a warp over with the group
walk when its stack would overflow. Natural inputs stay far below the stack's
capacity, so these runs shrink it (FLUXION_BH_BATCH_STACK, read once per
process) to send most warps, or some, down that path: per-point interaction
counts must still equal the oracle's and forces stay within 1e-5 of FP64."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

_SCRIPT = r"""
import sys
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import numpy as np
import fluxion_b200 as fx
from oracle import oracle as orc
orc.build()
rng = np.random.default_rng(int(sys.argv[3]))
n = 30000
centers = rng.random((12, 2)) * 400
pick = rng.integers(0, 12, n)
pts = (centers[pick] + rng.normal(0, 6.0, (n, 2))).clip(0, 400).astype(np.float32)
x, y = pts[:, 0].copy(), pts[:, 1].copy()
ctx = fx.Context(0)
d = fx.Design(ctx, fx.Circuit.from_nets([[0, 1]], n, 400.0, 400.0))
d.set_positions(x, y)
qx, qy, keys, perm, root, terms = d.barnes_hut(0.5, 0.5, 0.1, walk=fx.FX_BH_FAST, terms=True)
d.close()
ctx.close()
o = orc.bh_forces(x, y, 0.5, 0.5, float(np.float32(0.1)))
assert np.array_equal(keys, o["keys"]) and np.array_equal(perm, o["perm"])
assert np.array_equal(terms, o["interactions"]), "interaction counts differ"
num = np.sqrt(((qx - o["fx"]) ** 2 + (qy - o["fy"]) ** 2).sum())
err = num / np.sqrt((o["fx"] ** 2 + o["fy"] ** 2).sum())
assert err < 1e-5, err
print("fallback ok", err)
"""


@pytest.mark.parametrize("cap", [8, 96])
def test_batched_walk_overflow_fallback(fx, cap):
    env = dict(os.environ, FLUXION_BH_BATCH_STACK=str(cap), PYTHONFAULTHANDLER="1")
    r = subprocess.run([sys.executable, "-c", _SCRIPT, str(ROOT / "neon-physics-fluxion_b200"),
                        str(ROOT), str(cap)], capture_output=True, text=True, timeout=900,
                       env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fallback ok" in r.stdout
