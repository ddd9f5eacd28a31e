"""Build the CPU oracle ``oracle/liboracle.so`` (test infrastructure only).

gcc, FP contraction off so that FP32 neighbour membership follows the
explicit fmaf pattern of the restatement, OpenMP over particles.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    src = HERE / "vtp_oracle.c"
    hdr = HERE / "vtp_oracle.h"
    if not force and OUT.exists() and OUT.stat().st_mtime >= max(src.stat().st_mtime, hdr.stat().st_mtime):
        return OUT
    cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", str(OUT), str(src), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    try:
        print(build(force="--force" in sys.argv))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
