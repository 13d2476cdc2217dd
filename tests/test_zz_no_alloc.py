"""fx_congestion_noalloc, the congestion entry point that allocates no device
memory (its scratch is a fixed array inside the library), against
fx_congestion on the same inputs. Two calls in a row with different grids:
the second runs on the scratch the first left behind. Device buffers for the
inputs and outputs come from torch, as a caller's own pool would provide
them."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_noalloc(torch, d, cols, rows, x=None, y=None, outputs=True):
    dev = torch.device("cuda", 0)
    counts = torch.zeros(rows * cols, dtype=torch.int32, device=dev)  # uint32 bits
    res = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    mx = torch.full((1,), -1.0, dtype=torch.float32, device=dev)
    dx = torch.from_numpy(x).to(dev) if x is not None else None
    dy = torch.from_numpy(y).to(dev) if y is not None else None
    torch.cuda.synchronize()
    d.congestion_noalloc(cols, rows, counts.data_ptr(),
                         dx.data_ptr() if dx is not None else 0,
                         dy.data_ptr() if dy is not None else 0,
                         res.data_ptr() if outputs else 0, mx.data_ptr() if outputs else 0)
    d.ctx.synchronize()
    return (counts.cpu().numpy().view(np.uint32), float(res[0]), float(res[1]), float(mx[0]))


def test_noalloc_matches_fx_congestion_on_two_calls(fx, ctx, plain_small):
    import torch
    c = plain_small.circuit
    d = fx.Design(ctx, c)
    rng = np.random.default_rng(11)
    try:
        for cols, rows in [(64, 64), (97, 41)]:
            x = rng.uniform(0.0, c.chip_width, c.num_gates).astype(np.float32)
            y = rng.uniform(0.0, c.chip_height, c.num_gates).astype(np.float32)
            counts, hp, tot, mx = d.congestion(cols, rows, x, y)
            got, ghp, gtot, gmx = _run_noalloc(torch, d, cols, rows, x, y)
            assert np.array_equal(got, counts)
            assert (ghp, gtot, gmx) == (hp, tot, mx)
            assert counts.sum() > 0
    finally:
        d.close()


def test_noalloc_resident_positions_and_null_outputs(fx, ctx, plain_small):
    import torch
    c, p = plain_small.circuit, plain_small.placement
    d = fx.Design(ctx, c)
    try:
        d.set_positions(p.gate_x, p.gate_y)
        counts, hp, tot, mx = d.congestion(128, 96)
        got, ghp, gtot, gmx = _run_noalloc(torch, d, 128, 96)
        assert np.array_equal(got, counts) and (ghp, gtot, gmx) == (hp, tot, mx)
        # results kept in the scratch when the caller passes no result buffers
        got2 = _run_noalloc(torch, d, 128, 96, outputs=False)[0]
        assert np.array_equal(got2, counts)
    finally:
        d.close()


def test_noalloc_rejects_grids_beyond_its_scratch(fx, ctx, plain_small):
    import torch
    d = fx.Design(ctx, plain_small.circuit)
    try:
        out = torch.zeros(4, dtype=torch.int32, device="cuda")
        with pytest.raises(fx.FluxionError, match="scratch"):
            d.congestion_noalloc(1500, 1500, out.data_ptr())
        with pytest.raises(fx.FluxionError):
            d.congestion_noalloc(64, 64, 0)  # no count buffer
    finally:
        d.close()


_FRESH = r"""
import sys
import numpy as np
import torch
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import fluxion_b200 as fx
fx.load()
s = fx.synth_plain(7, 4000, 4800, 76.0)
c = s.circuit
dev = torch.device("cuda", 0)
# torch.empty and host-to-device copies launch no kernel: the no-alloc call
# below is the first kernel work of this process on the device
counts = torch.empty(64 * 64, dtype=torch.int32, device=dev)
res = torch.empty(2, dtype=torch.float64, device=dev)
mx = torch.empty(1, dtype=torch.float32, device=dev)
dx = torch.from_numpy(s.placement.gate_x).to(dev)
dy = torch.from_numpy(s.placement.gate_y).to(dev)
torch.cuda.synchronize()
ctx = fx.Context(0)
d = fx.Design(ctx, c)
d.congestion_noalloc(64, 64, counts.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                     res.data_ptr(), mx.data_ptr())
ctx.synchronize()
got = counts.cpu().numpy().view(np.uint32)
want, hp, tot, m = d.congestion(64, 64, s.placement.gate_x, s.placement.gate_y)
assert want.sum() > 0
assert np.array_equal(got, want), "first no-alloc call differs"
assert (float(res[0]), float(res[1]), float(mx[0])) == (hp, tot, m)
d.close()
ctx.close()
print("fresh ok")
"""


def test_noalloc_first_call_in_a_fresh_process(fx):
    """The scratch set-up and the first call's kernels in a process whose
    device has run nothing else: the zeroing must be ordered before them."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, "-c", _FRESH, str(root / "neon-physics-fluxion_b200"),
                        str(root)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh ok" in r.stdout
