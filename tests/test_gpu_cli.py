"""The `fluxion` command and FluxionEngine end to end on the GPU: a BLIF in,
a DEF out (the reference's integration test, H/tests/test_integration.py),
with the same coordinates as the library pipeline called step by step."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _random_blif(path: Path, n: int, seed: int) -> None:
    rng = np.random.default_rng(seed)
    lines = [".model rnd", ".inputs " + " ".join(f"i{k}" for k in range(16)), ".outputs o"]
    sig = [f"i{k}" for k in range(16)]
    for g in range(n):
        k = int(rng.integers(1, 4))
        ins = [sig[int(j)] for j in rng.integers(max(0, len(sig) - 200), len(sig), k)]
        out = f"w{g}"
        if g % 7 == 0:
            lines.append(f".gate G{k} " + " ".join(f"a{j}={s}" for j, s in enumerate(ins)) +
                         f" O={out}")
        elif g % 11 == 0:
            lines.append(f".latch {ins[0]} {out}")
        else:
            lines.append(".names " + " ".join(ins) + f" {out}")
            lines.append("1" * k + " 1")
        sig.append(out)
    lines.append(".end")
    path.write_text("\n".join(lines) + "\n")


def _def_coords(text: str):
    rows = re.findall(r"- (\S+) GATE_TYPE \+ PLACED \( (-?\d+) (-?\d+) \) N ;", text)
    return [r[0] for r in rows], np.array([[int(r[1]), int(r[2])] for r in rows], np.int64)


def test_cli_places_a_blif_like_the_library(fx, ctx, tmp_path):
    blif = tmp_path / "rnd.blif"
    _random_blif(blif, 3000, 5)
    out = tmp_path / "rnd.def"
    r = subprocess.run([str(fx.engine.BINARY), "--config", str(fx.engine.DEFAULT_CONFIG),
                        "--input", str(blif), "--output", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Done! HPWL" in r.stderr
    text = out.read_text()
    assert "COMPONENTS 3000 ;" in text and "END COMPONENTS" in text and "+ PLACED" in text
    assert "DESIGN rnd ;" in text and "DIEAREA ( 0 0 ) ( 1000000 1000000 ) ;" in text
    names, xy = _def_coords(text)
    assert names == [f"g{i}" for i in range(3000)]
    assert xy.min() >= 0 and xy.max() <= 1_000_000
    # the same flow through the library
    c = fx.read_blif(blif)
    d = fx.Design(ctx, c)
    try:
        t = d.partition(fx.part_cfg())
        x, y, _ = d.place_leaves(t["leaf_ptr"], t["leaf_gate"], t["region"].reshape(-1),
                                 fx.leaf_cfg())
        d.refine(fx.refine_cfg(), x, y)
    finally:
        d.close()
    ref = tmp_path / "lib.def"
    fx.write_def(ref, c, fx.Placement(x, y))
    assert ref.read_text() == text


def test_engine_place(fx, tmp_path, capsys):
    blif = tmp_path / "e.blif"
    _random_blif(blif, 500, 9)
    eng = fx.FluxionEngine(str(fx.engine.DEFAULT_CONFIG))
    out = eng.place(str(blif), str(tmp_path / "e.def"))
    assert Path(out).exists() and "+ PLACED" in Path(out).read_text()
    assert "Placement saved" in capsys.readouterr().out
