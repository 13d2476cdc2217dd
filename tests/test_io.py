"""Netlist ingestion (BLIF) and DEF output, host-only; the `fluxion` command's
argument, config and input checks (exit codes of H/src/main.rs, before any GPU
work); FluxionEngine's errors."""
from __future__ import annotations

import os

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _nets(c):
    return [c.net_gate[c.net_ptr[e]:c.net_ptr[e + 1]].tolist() for e in range(c.num_nets)]


def test_blif_reader_follows_the_reference_rules(fx):
    c = fx.read_blif(GOLDEN / "io_mixed.blif")
    # gates in line order: g0 .names w1, g1 .gate Y=w2, g2 .latch w3, g3 .gate O=s,
    # g4 .names t, g5 .gate O=w4, g6 .names w5 (no inputs)
    assert c.num_gates == 7 and c.name == "io_mixed"
    assert c.gate_names == [f"g{i}" for i in range(7)]
    assert np.all(c.gate_widths == 2.0) and np.all(c.gate_heights == 10.0)
    assert (c.chip_width, c.chip_height) == (1000.0, 1000.0)
    # driven signals first (w1, w2, w3, s, t, w4, w5), each driver then its
    # readers; then undriven signals read by >= 2 gates (p, r); one-gate nets
    # (s, t, w4, w5, q) are dropped
    assert _nets(c) == [[0, 1, 4], [1, 2], [2, 3, 4], [0, 5], [1, 5]]


# the reference project's root, when a checkout is at hand (FLUXION_REFERENCE)
_REF = os.environ.get("FLUXION_REFERENCE", "")
REF_SMALL_BLIF = Path(_REF, "HAPR_fluxion_v4", "tests", "fixtures", "small.blif") if _REF else None


@pytest.mark.skipif(REF_SMALL_BLIF is None or not REF_SMALL_BLIF.exists(),
                    reason="FLUXION_REFERENCE does not name a reference checkout")
def test_blif_reader_on_the_reference_fixture(fx):
    """The reference's end-to-end fixture (tests/test_integration.py:10-38
    places it), read where it lies: four .gate lines (AND2 a b -> n1, OR2 c d
    -> n2, XOR2 n1 n2 -> y, INV n2 -> z). By blif.rs:88-116 the driven nets
    n1 = {g0, g2} and n2 = {g1, g2, g3} remain; y, z and the primary inputs
    touch one gate each and are dropped."""
    c = fx.read_blif(REF_SMALL_BLIF)
    assert c.num_gates == 4 and c.name == "small"
    assert _nets(c) == [[0, 2], [1, 2, 3]]


def test_blif_reader_rejects_missing_file(fx):
    with pytest.raises(fx.FluxionError, match="open BLIF"):
        fx.read_blif("/nonexistent/x.blif")


def test_def_writer_format_and_rounding(fx, tmp_path):
    c = fx.Circuit.from_nets([[0, 1], [1, 2]], 3, chip_width=12.5, chip_height=7.25,
                             name="tiny", gate_names=["a", "b", "c"])
    p = fx.Placement(np.array([1.2345, -0.0015, np.nan], np.float32),
                     np.array([0.0, 6.9999, 1e30], np.float32))
    out = tmp_path / "t.def"
    fx.write_def(out, c, p)
    want = ("VERSION 5.8 ;\nDIVIDERCHAR \"/\" ;\nBUSBITCHARS \"[]\" ;\nDESIGN tiny ;\n"
            "UNITS DISTANCE MICRONS 1000 ;\n\nDIEAREA ( 0 0 ) ( 12500 7250 ) ;\n\n"
            "COMPONENTS 3 ;\n"
            f"    - a GATE_TYPE + PLACED ( {int(np.float32(1.2345) * np.float32(1000))} 0 ) N ;\n"
            f"    - b GATE_TYPE + PLACED ( -1 {int(np.float32(6.9999) * np.float32(1000))} ) N ;\n"
            "    - c GATE_TYPE + PLACED ( 0 9223372036854775807 ) N ;\n"
            "END COMPONENTS ;\n\nEND DESIGN\n")
    assert out.read_text() == want


def _cli(fx, *args, cwd=None):
    b = Path(fx.engine.BINARY)
    r = subprocess.run([str(b), *args], capture_output=True, text=True, cwd=cwd, timeout=60)
    return r.returncode, r.stdout, r.stderr


def test_cli_arguments_and_input_checks(fx, tmp_path):
    cfg = Path(fx.engine.DEFAULT_CONFIG)
    rc, out, _ = _cli(fx, "--help")
    assert rc == 0 and "--config" in out
    assert _cli(fx, "--bogus")[0] == 2
    assert _cli(fx, "--config")[0] == 2
    rc, _, err = _cli(fx, "--config", str(tmp_path / "none.yaml"))
    assert rc == 1 and "Config error" in err
    rc, _, err = _cli(fx, "--config", str(cfg))  # input: "" in the defaults
    assert rc == 1 and "No input file" in err
    rc, _, err = _cli(fx, "--config", str(cfg), "--input", str(tmp_path / "x.def"))
    assert rc == 1 and "Unsupported format" in err
    rc, _, err = _cli(fx, "--config", str(cfg), "--input", str(tmp_path / "missing.blif"))
    assert rc == 1 and "BLIF parse error" in err
    empty = tmp_path / "empty.blif"
    empty.write_text(".model e\n.inputs a\n.end\n")
    rc, _, err = _cli(fx, "--config", str(cfg), "--input", str(empty))
    assert rc == 1 and "0 gates" in err
    broken = tmp_path / "broken.yaml"
    broken.write_text(cfg.read_text().replace("  dt: 0.1\n", ""))
    rc, _, err = _cli(fx, "--config", str(broken), "--input", str(empty))
    assert rc == 1 and "placement.dt" in err
    bad = tmp_path / "bad.yaml"
    bad.write_text(cfg.read_text().replace("max_leaf_size: 64", "max_leaf_size: -3"))
    rc, _, err = _cli(fx, "--config", str(bad), "--input", str(empty))
    assert rc == 1 and "expected usize" in err


def test_engine_errors(fx, tmp_path):
    with pytest.raises(FileNotFoundError):
        fx.FluxionEngine(str(tmp_path / "nope.yaml"))
    eng = fx.FluxionEngine(str(fx.engine.DEFAULT_CONFIG))
    assert eng.config["partitioning"]["max_leaf_size"] == 64
    with pytest.raises(FileNotFoundError):
        eng.place(str(tmp_path / "nope.blif"))
