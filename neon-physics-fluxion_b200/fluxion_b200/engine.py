"""FluxionEngine: the reference's Python entry point (H/python/fluxion/engine.py)
over this library. `place` runs the `fluxion` command (the reference ran
`cargo run --release -- ...`; there is no cargo here), with the same
arguments, output and errors."""
from __future__ import annotations

import subprocess
from pathlib import Path

import yaml

PKG = Path(__file__).resolve().parent
BINARY = PKG / "fluxion"
DEFAULT_CONFIG = PKG.parent / "config" / "default.yaml"


def _require(path: Path, what: str) -> Path:
    if not path.exists():
        raise FileNotFoundError(f"{what}: {path}")
    return path


class FluxionEngine:
    """Places a BLIF netlist with the HAPR flow on the GPU.

    The YAML configuration is parsed once when the engine is made (a missing
    file raises FileNotFoundError) and kept in `config`. Each `place` call
    hands the configuration file, the netlist and the output path to the
    `fluxion` command built next to this module, which writes a DEF file.
    """

    def __init__(self, config_path="default.yaml"):
        self.config_path = _require(Path(config_path), "Config not found")
        self.config = yaml.safe_load(self.config_path.read_text())

    def _command(self, netlist: Path, output_file) -> list[str]:
        if not BINARY.exists():
            raise FileNotFoundError(f"{BINARY} is missing; build it with "
                                    "`python -c 'import __graft_entry__ as g; g.build()'`")
        return [str(BINARY), "--config", str(self.config_path), "--input", str(netlist),
                "--output", str(output_file)]

    def place(self, input_file: str, output_file: str = "placed.def"):
        """Returns `output_file` once the command has written it; a non-zero
        exit of the command prints its stderr and raises RuntimeError."""
        cmd = self._command(_require(Path(input_file), "Input file not found"), output_file)
        print(f"Running FLUXION core: {' '.join(cmd)}")
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode == 0:
            print(proc.stdout)
            print(f"Placement saved to {output_file}")
            return output_file
        print("FLUXION Core Error:")
        print(proc.stderr)
        raise RuntimeError("Placement failed")
