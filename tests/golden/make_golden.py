"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run where a checkout of the reference project is at hand, named by the
FLUXION_REFERENCE environment variable (it reads the reference sources;
nothing at test time does):

    FLUXION_REFERENCE=<reference checkout> python tests/golden/make_golden.py

* golden_dct.npz -- the reference's own ElectrostaticSmoothingForce
  (neon_old_codebase/src/python/fluxion/force_electrostatic.py) on seeded
  particles: _solve_poisson_fft on seeded charge grids (G = 64, 128) and
  calculate() forces / energy on 1500 particles (G = 64).
* golden_bh.npz -- forces from the reference's own Barnes-Hut tree
  (neon_old_codebase/src/cpp/BarnesHutTree.cpp, compiled into oracle/_ref by
  oracle/Makefile) on seeded point sets, theta = 0.5 and theta = 0.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_ROOT = Path(os.environ.get("FLUXION_REFERENCE", ""))
REF_PY = REF_ROOT / "neon_old_codebase" / "src" / "python"


def dct_fixtures(out: dict) -> None:
    sys.path.insert(0, str(REF_PY))
    from fluxion.force_electrostatic import ElectrostaticSmoothingForce
    from fluxion.particle_system import FluxionParticle, FluxionParticleSystem

    rng = np.random.default_rng(7)
    for G in (64, 128):
        rho = rng.normal(0.0, 1.0, (G, G))
        f = ElectrostaticSmoothingForce(weight=1.0, grid_size=G, target_density=0.7)
        wx, wy = G / 100.0, G / 80.0
        phi, ex, ey = f._solve_poisson_fft(rho, wx, wy)
        out[f"solve{G}_rho"] = rho
        out[f"solve{G}_w"] = np.array([wx, wy])
        out[f"solve{G}_phi"] = phi
        out[f"solve{G}_ex"] = ex
        out[f"solve{G}_ey"] = ey
    # calculate(): 1500 particles on a 100 x 100 die, G = 64 (bin 1.5625,
    # exact in binary, so f32 and f64 bins agree for f32 positions).
    G, die, n = 64, 100.0, 1500
    xs = (rng.random(n) * die).astype(np.float32)
    ys = (rng.random(n) * die).astype(np.float32)
    area = rng.integers(1, 5, n).astype(np.float64)
    bw = die / G
    assert np.array_equal(np.clip(xs.astype(np.float64) / bw, 0, G - 1).astype(int),
                          np.clip(xs / np.float32(bw), 0, G - 1).astype(int))
    system = FluxionParticleSystem(die_width=die, die_height=die)
    for i in range(n):
        system.add_particle(FluxionParticle(id=i, name=f"g{i}", type="NAND",
                                            x=float(xs[i]), y=float(ys[i]),
                                            area_um2=float(area[i])))
    f = ElectrostaticSmoothingForce(weight=1.0, grid_size=G, target_density=0.7)
    res = f.calculate(system)
    out["calc_x"], out["calc_y"], out["calc_area"] = xs, ys, area
    out["calc_meta"] = np.array([G, die, 0.7, 1.0])
    out["calc_forces"] = res.forces
    out["calc_energy"] = np.array([res.energy])


def bh_fixtures(out: dict) -> None:
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as orc

    orc.build()
    rng = np.random.default_rng(11)
    sets = {
        "uniform": (rng.random((3000, 2)) * 100.0).astype(np.float32),
        "clustered": np.concatenate([
            (rng.normal(c, 3.0, (600, 2))).astype(np.float32)
            for c in ((20, 20), (70, 30), (50, 80), (85, 85), (10, 90))]),
        "small": (rng.random((200, 2)) * 10.0).astype(np.float32),
    }
    for name, pts in sets.items():
        x, y = pts[:, 0].copy(), pts[:, 1].copy()
        out[f"bh_{name}_x"], out[f"bh_{name}_y"] = x, y
        for theta in (0.5, 0.0):
            fx, fy = orc.bh_reference(x, y, k=0.5, theta=theta, min_dist=0.1)
            tag = "t05" if theta else "t0"
            out[f"bh_{name}_{tag}_fx"] = fx
            out[f"bh_{name}_{tag}_fy"] = fy


def main() -> None:
    if not (REF_PY / "fluxion").is_dir():
        sys.exit("set FLUXION_REFERENCE to a checkout of the reference project")
    dct: dict = {}
    dct_fixtures(dct)
    np.savez_compressed(HERE / "golden_dct.npz", **dct)
    bh: dict = {}
    bh_fixtures(bh)
    np.savez_compressed(HERE / "golden_bh.npz", **bh)
    for p in ("golden_dct.npz", "golden_bh.npz"):
        print(p, (HERE / p).stat().st_size, "bytes")


if __name__ == "__main__":
    main()
