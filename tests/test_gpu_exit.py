"""A script that leaves its context and design open exits cleanly: the
package closes open handles (designs before their contexts) when the
interpreter exits, after cached CUDA graphs of single-iteration calls were
replayed and stage timing was switched on and off."""
import pytest

pytestmark = pytest.mark.gpu

_SCRIPT = r"""
import sys
sys.path[:0] = [sys.argv[1]]
import fluxion_b200 as fx
s = fx.synth_plain(21, 8000, 9600, 108.0)
ctx = fx.Context(0)
d = fx.Design(ctx, s.circuit)
cfg = fx.iter_cfg(density_bins=128, cong_cols=32, cong_rows=32)
d.set_positions(s.placement.gate_x, s.placement.gate_y)
d.save_state()
for _ in range(8):  # eager, captured, then replayed calls
    d.restore_state()
    st = d.force_iterate(cfg, 1)
ctx.set_profiling(True)
for _ in range(2):
    d.restore_state()
    st = d.force_iterate(cfg, 1)
ctx.synchronize()
ctx.set_profiling(False)
print("left open", st.hpwl > 0)
"""


def test_open_handles_at_exit(fx):
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, PYTHONFAULTHANDLER="1")  # a crash prints where it was
    r = subprocess.run([sys.executable, "-c", _SCRIPT, str(root / "neon-physics-fluxion_b200")],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "left open True" in r.stdout
