"""Fixed-form Fortran 77 source reader.

Turns a fixed-form source file into logical statements: comment lines
(``C``, ``c``, ``*``, ``!`` in column 1) are dropped, continuation lines
(non-blank, non-zero column 6) are joined, columns beyond 72 are ignored,
and a leading TAB starts the statement field (DEC tab format, which the
UNICORN sources use in a few places, e.g. ``unicornd-mild-sd-5.f:471-483``).

Each logical statement keeps the 1-based line number of its first physical
line and its numeric label, so that callers can select line ranges and
resolve ``GO TO`` targets.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class RawStatement:
    line: int          # 1-based line number of the first physical line
    last_line: int     # 1-based line number of the last continuation line
    label: int | None  # statement label (columns 1-5), if any
    text: str          # statement text, columns 7-72 joined, blanks kept


def _expand(line: str) -> str:
    """Expand a physical line to fixed columns (TAB in columns 1-6 -> col 7)."""
    line = line.rstrip("\r\n")
    head = line[:6]
    if "\t" in head:
        k = line.index("\t")
        lab = line[:k]
        rest = line[k + 1:]
        # DEC convention: TAB followed by a digit 1-9 is a continuation line.
        if rest[:1].isdigit() and rest[:1] != "0":
            return lab.ljust(5)[:5] + rest[0] + rest[1:].replace("\t", " ")
        return lab.ljust(6)[:6] + rest.replace("\t", " ")
    return line.replace("\t", " ")


def read_fixed_form(path: str) -> list[RawStatement]:
    with open(path, "r", encoding="latin-1") as fh:
        physical = fh.readlines()
    out: list[RawStatement] = []
    cur: RawStatement | None = None
    for lineno, raw in enumerate(physical, start=1):
        if not raw.strip():
            continue
        if raw[0] in "Cc*!":
            continue
        line = _expand(raw)
        if not line.strip():
            continue
        label_field = line[:5]
        cont = line[5:6]
        body = line[6:72]
        if cont not in ("", " ", "0"):
            if cur is None:
                raise ValueError(f"{path}:{lineno}: continuation without statement")
            cur.text += body
            cur.last_line = lineno
            continue
        if cur is not None:
            out.append(cur)
        lab = label_field.strip()
        cur = RawStatement(lineno, lineno, int(lab) if lab else None, body)
    if cur is not None:
        out.append(cur)
    return out
