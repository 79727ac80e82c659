"""The C ABI library loads here (no GPU needed) and exports what ``include/bt200.h`` declares."""

from __future__ import annotations

import re
from pathlib import Path

from beamtracer_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "bt200.h"


def _declared() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(bt_[a-z0-9_]+)\s*\(", text))


def test_every_declared_entry_point_is_exported_and_bound():
    declared = _declared()
    assert declared, "no entry points parsed from the header"
    handle = _lib.lib()
    for name in sorted(declared):
        assert hasattr(handle, name), f"{name} is declared but not exported"
    assert declared == set(_lib.exported_symbols())


def test_version_and_error_buffer():
    assert b"sm_100a" in _lib.lib().bt_version()
    assert isinstance(_lib.last_error(), str)
