"""FluxionEngine: the reference's Python entry point (H/python/fluxion/engine.py)
on this build. `place` runs the `fluxion` command (the reference ran
`cargo run --release -- ...`; there is no cargo here), with the same
arguments, output and errors."""
from __future__ import annotations

import subprocess
from pathlib import Path

import yaml

PKG = Path(__file__).resolve().parent
BINARY = PKG / "fluxion"
DEFAULT_CONFIG = PKG.parent / "config" / "default.yaml"


class FluxionEngine:
    """
    Usage:
        engine = FluxionEngine("config/default.yaml")
        engine.place("circuit.blif")
    """

    def __init__(self, config_path="default.yaml"):
        self.config_path = Path(config_path)
        if not self.config_path.exists():
            raise FileNotFoundError(f"Config not found: {self.config_path}")
        with open(self.config_path, "r") as f:
            self.config = yaml.safe_load(f)

    def place(self, input_file: str, output_file: str = "placed.def"):
        """Runs the full HAPR flow on the GPU through the `fluxion` command."""
        input_path = Path(input_file)
        if not input_path.exists():
            raise FileNotFoundError(f"Input file not found: {input_path}")
        if not BINARY.exists():
            raise FileNotFoundError(f"{BINARY} is missing; build it with "
                                    "`python -c 'import __graft_entry__ as g; g.build()'`")
        cmd = [str(BINARY), "--config", str(self.config_path), "--input", str(input_path),
               "--output", str(output_file)]
        print(f"Running FLUXION core: {' '.join(cmd)}")
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            print("FLUXION Core Error:")
            print(result.stderr)
            raise RuntimeError("Placement failed")
        print(result.stdout)
        print(f"Placement saved to {output_file}")
        return output_file
