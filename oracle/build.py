"""ORACLE build recipe (test infrastructure): compile the C restatement into a shared library.

``python -m oracle.build`` (or `build()`) runs gcc on ``oracle/bt_oracle.c`` and writes
``oracle/_build/libbt_oracle.so``.  No multiply-add is fused (``-ffp-contract=off``), so the
library rounds exactly as the expressions are written; OpenMP splits the trace over host
threads as the reference's Pyccel build does.
"""

from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "bt_oracle.c"
LIBRARY = HERE / "_build" / "libbt_oracle.so"


def build(force: bool = False) -> Path:
    """Compile the oracle library if it is missing or older than its source; return its path."""
    if (
        not force
        and LIBRARY.exists()
        and LIBRARY.stat().st_mtime >= SOURCE.stat().st_mtime
    ):
        return LIBRARY
    LIBRARY.parent.mkdir(parents=True, exist_ok=True)
    command = [
        "gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp",
        "-ffp-contract=off", "-fno-fast-math",
        str(SOURCE), "-o", str(LIBRARY), "-lm",
    ]  # fmt: skip
    subprocess.run(command, check=True)
    return LIBRARY


if __name__ == "__main__":
    print(build(force=True))
