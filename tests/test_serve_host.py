"""Host-only parts of the server: the admission estimate (no GPU)."""
from __future__ import annotations

import numpy as np


def test_estimates_grow_with_the_design(fx):
    small = fx.synth_plain(1, 5_000, 6_000, 85.0).circuit
    large = fx.synth_plain(1, 50_000, 60_000, 268.0).circuit
    es = fx.serve_estimate(fx.Server.place_desc(small))
    el = fx.serve_estimate(fx.Server.place_desc(large))
    assert 0 < es < el
    # at least the netlist, adjacency and positions it must hold
    assert el > 4 * large.num_pins + 24 * large.num_gates
    e1 = fx.serve_estimate(fx.Server.eco_desc(1, np.arange(10), np.zeros(10), np.zeros(10),
                                              n_gates=5_000))
    e2 = fx.serve_estimate(fx.Server.eco_desc(1, np.arange(10), np.zeros(10), np.zeros(10),
                                              n_gates=500_000))
    assert 0 < e1 < e2


def test_invalid_job_is_rejected(fx):
    import pytest
    d, keep = fx.Server.eco_desc(1, np.arange(3), np.zeros(3), np.zeros(3), iterations=-1)
    with pytest.raises(fx.FluxionError):
        fx.serve_estimate((d, keep))
