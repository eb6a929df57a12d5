"""Times the surrogate's tcgen05 convolutions (forward, input gradient, weight gradient) on an
N x H x W batch of 64-channel activations and prints JSON.

    python -m fip_b200.conv_cli [--N 32 --H 512 --W 512 --iters 20]
"""
from __future__ import annotations

import argparse
import json

from .surrogate import bench_convs


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=32)
    ap.add_argument("--H", type=int, default=512)
    ap.add_argument("--W", type=int, default=512)
    ap.add_argument("--iters", type=int, default=20)
    a = ap.parse_args(argv)
    print(json.dumps(bench_convs(a.N, a.H, a.W, a.iters)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
