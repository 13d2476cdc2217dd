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
