"""Where the reference checkout (UNICORN's Fortran sources) is read from.

Only the recipes that translate or extract from the reference use this: the
mechanism extractor, the reference build recipe under oracle/ and the tests
that read the reference's text. The library itself never reads it.

The location is the environment variable UNICORN_REF, else a directory named
``reference`` beside this repository's root.
"""
from __future__ import annotations

import os
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def reference_root() -> Path:
    env = os.environ.get("UNICORN_REF")
    return Path(env) if env else REPO.parent / "reference"
