"""Build recipe for the oracle libraries (test infrastructure).

``serial.c`` (the reference's serial engine restated) and ``replay.c`` (a
host replay of the device sweep's schedule) compile with gcc into
``oracle/_build/liboracle.so``. Run ``python -m oracle.build`` or call
``build()``; both are no-ops when the library is newer than its sources.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build"
LIB = OUT / "liboracle.so"
SOURCES = [HERE / "serial.c", HERE / "replay.c"]

# No fused multiply-add anywhere: the serial engine is pinned bit for bit to
# the reference's f64 arithmetic, and the replay to the device's own
# operation order, where every fusion is written out explicitly.
CFLAGS = ["-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-fvisibility=hidden"]


def build(force: bool = False) -> Path:
    sources = [s for s in SOURCES if s.exists()]
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return LIB
    OUT.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", *CFLAGS, "-o", str(tmp), *map(str, sources), "-lm"]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
