"""The C-ABI library loads and exports every declared symbol; host-only entry
points (the synthetic generator) work without a GPU."""
import re
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fluxion_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fx_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("fx_ctx_create", "fx_design_load", "fx_congestion", "fx_force_iterate",
                 "fx_stage_barnes_hut", "fx_stage_density"):
        assert must in names


def test_library_exports_every_declared_symbol(fx):
    from fluxion_b200 import _lib
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (fx_[a-z0-9_]+)$", out, flags=re.M))
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_context_without_device_is_refused(fx):
    import ctypes as C
    from fluxion_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.fx_ctx_create(C.byref(h), 0)
    if rc == _lib.FX_OK:  # a GPU is present: creation works
        lib.fx_ctx_destroy(h)
    else:
        assert rc == _lib.FX_ENODEV
        assert lib.fx_last_error()


def test_invalid_arguments_are_rejected(fx):
    import ctypes as C
    from fluxion_b200 import _lib
    lib = _lib.load()
    assert lib.fx_ctx_create(None, 0) == _lib.FX_EINVAL
    assert lib.fx_design_load(None, 0, 0, None, None, None, None, 1.0, 1.0,
                              None) == _lib.FX_EINVAL
    h = C.c_void_p()
    assert lib.fx_synth_plain(1, 0, 10, 10.0, 10.0, 64, C.byref(h)) == _lib.FX_EINVAL


def test_synth_plain_shape_and_determinism(fx):
    a = fx.synth_plain(42, 10_000, 12_000, 120.0)
    b = fx.synth_plain(42, 10_000, 12_000, 120.0)
    c = a.circuit
    assert np.array_equal(c.net_gate, b.circuit.net_gate)
    assert np.array_equal(a.placement.gate_x, b.placement.gate_x)
    deg = np.diff(c.net_ptr)
    assert c.num_nets == 12_000 and deg.min() >= 2 and deg.max() <= 64
    assert 0.55 < np.mean(deg == 2) < 0.72  # 0.6 plus the power-law mass at 2
    assert 2.4 < deg.mean() < 2.9           # ~2.6 pins per net
    assert c.net_gate.min() >= 0 and c.net_gate.max() < 10_000
    for e in range(0, 12_000, 97):
        pins = c.net_gate[c.net_ptr[e]:c.net_ptr[e + 1]]
        assert len(set(pins.tolist())) == len(pins)
    x, y = a.placement.gate_x, a.placement.gate_y
    assert x.min() >= 0 and x.max() < 120 and y.min() >= 0 and y.max() < 120
    assert set(np.unique(c.gate_widths).tolist()) == {1.0, 2.0, 3.0, 4.0}
    # pins stay local: most pins share the driver's leaf or its sibling
    drv_leaf = c.net_gate[c.net_ptr[:-1]] // 64
    owner = np.repeat(drv_leaf, deg)
    pl = c.net_gate // 64
    assert np.mean((pl == owner) | (pl == (owner ^ 1))) > 0.85


def test_synth_leaves_shape(fx):
    s = fx.synth_leaves(7, 256, 16, 128, 1.5)
    sizes = np.diff(s.leaf_ptr)
    assert len(sizes) == 256 and sizes.min() >= 16 and sizes.max() <= 128
    c = s.circuit
    deg = np.diff(c.net_ptr)
    assert deg.min() >= 2 and deg.max() <= 8
    # every net stays inside one cluster
    leaf_of = np.repeat(np.arange(256), sizes)
    first = leaf_of[c.net_gate[c.net_ptr[:-1]]]
    assert np.all(leaf_of[c.net_gate] == np.repeat(first, deg))
    assert abs(c.num_nets / c.num_gates - 1.5) < 0.02


def test_adjacency_order_matches_reference(fx, oracle):
    # circuit.rs:154-171: the product's host builder reproduces the reference's
    # lists in insertion order, including nets that name a gate twice.
    s = fx.synth_plain(5, 3000, 3600, 60.0)
    ap, ai = fx.build_adjacency(s.circuit)
    rp, ri = oracle.build_adjacency(3000, s.circuit.net_ptr, s.circuit.net_gate)
    assert np.array_equal(ap, rp) and np.array_equal(ai, ri)
    nets = [[0, 1, 0, 2], [2, 2], [3, 1, 3, 3, 0], [4], [], [1, 4, 1]]
    c = fx.Circuit.from_nets(nets, 5)
    ap, ai = fx.build_adjacency(c)
    rp, ri = oracle.build_adjacency(5, c.net_ptr, c.net_gate)
    assert np.array_equal(ap, rp) and np.array_equal(ai, ri)


def test_adjacency_rejects_bad_csr(fx):
    import pytest
    c = fx.Circuit.from_nets([[0, 7]], 3)
    with pytest.raises(fx.FluxionError):
        fx.build_adjacency(c)


def test_python_constants_match_the_header():
    """Every FX_* integer constant of the ctypes mirror equals the header's
    #define of the same name, and the header's schedule, precision, stage,
    status and job codes all have a Python twin."""
    from fluxion_b200 import _lib
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    defines = {k: int(v) for k, v in re.findall(r"#define\s+(FX_[A-Z0-9_]+)\s+(-?\d+)\b", text)}
    mirrored = {k: v for k, v in vars(_lib).items() if k.startswith("FX_") and isinstance(v, int)}
    assert mirrored
    for k, v in mirrored.items():
        assert k in defines and defines[k] == v, k
    for k in defines:
        if k.startswith(("FX_LEAF_", "FX_DCT_", "FX_PART_", "FX_JOB_", "FX_E")):
            assert k in mirrored, k
    # stage codes index the STAGES name list
    stages = {k[len("FX_STAGE_"):].lower(): v for k, v in defines.items()
              if k.startswith("FX_STAGE_") and k != "FX_STAGE_COUNT"}
    assert len(_lib.STAGES) == defines["FX_STAGE_COUNT"] == len(stages)
    for name, code in stages.items():
        assert _lib.STAGES[code] == name, name


def test_exit_hook_closes_designs_and_servers_before_contexts(fx):
    """The interpreter-exit hook closes every handle still open, designs and
    servers before the contexts they run on (order recorded on stand-ins)."""
    from fluxion_b200 import api
    closed = []

    class Stub:
        def __init__(self, kind):
            self.kind = kind

        def close(self):
            closed.append(self.kind)

    saved = {k: list(v) for k, v in api._OPEN.items()}
    stubs = [Stub("ctx"), Stub("design"), Stub("server"), Stub("design")]
    try:
        for k in api._OPEN:
            api._OPEN[k].clear()
        for st in stubs:
            api._OPEN[st.kind].add(st)
        api._close_open_handles()
    finally:
        for k in api._OPEN:
            api._OPEN[k].clear()
            for o in saved[k]:
                api._OPEN[k].add(o)
    assert closed == ["design", "design", "server", "ctx"]
