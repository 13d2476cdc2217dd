"""Shared pytest setup: import paths, the `gpu` marker and fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "neon-physics-fluxion_b200"
for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc
    orc.build()
    return orc


@pytest.fixture(scope="session")
def fx():
    import fluxion_b200
    fluxion_b200.load()
    return fluxion_b200


@pytest.fixture(scope="session")
def ctx(fx):
    c = fx.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def plain_small(fx):
    """The plain-small workload: 10,000 gates, 12,000 nets, die 120 x 120."""
    return fx.synth_plain(42, 10_000, 12_000, 120.0)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = ROOT / "tests" / "golden"
    return {"dct": np.load(d / "golden_dct.npz"), "bh": np.load(d / "golden_bh.npz")}
