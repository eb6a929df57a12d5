"""Re-create a golden case (tests/golden/*.npz) in a scratch directory."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


class Golden:
    def __init__(self, name: str):
        self.name = name
        self.d = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.meta = json.loads(str(self.d["meta"]))
        self.W, self.H = self.meta["W"], self.meta["H"]
        self.pitch_elems = self.meta["pitch_bytes"] // 4
        self.stdout = str(self.d["stdout"])

    def materialize(self, outdir: str) -> str:
        """Write the case's input files to `outdir`; returns the YAML path with paths rewritten."""
        os.makedirs(outdir, exist_ok=True)
        old = self.meta["workdir"]
        for k in self.d.files:
            if k.startswith("file:"):
                with open(os.path.join(outdir, k[5:]), "wb") as f:
                    f.write(self.d[k].tobytes())
        y = str(self.d["yaml"]).replace(old, outdir)
        path = os.path.join(outdir, self.name + ".yml")
        with open(path, "w") as f:
            f.write(y)
        return path

    def dump_times(self):
        return sorted({int(k.split("_")[-1]) for k in self.d.files if k.startswith("dump_ah_")})

    def dump(self, kind: str, t: int) -> np.ndarray:
        return self.d[f"dump_{kind}_{t}"]
