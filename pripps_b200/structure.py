"""Structures: positions and species ids of the scatterers.

Mirrors the reference's ``Structure{pos, ids}`` (src/structure.rs:27-31) with
numpy arrays — positions [N, 3] FP64 in Å and species ids [N] indexing a
``FormFactorMap`` — and its lenient XYZ reader (src/input.rs:143-170).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .errors import ValidationError
from .formfactor import FormFactorMap


@dataclass
class Structure:
    pos: np.ndarray                      # [N, 3] float64, Å
    ids: np.ndarray                      # [N] int, species ids
    box_sides: Optional[np.ndarray] = None

    def __post_init__(self):
        self.pos = np.ascontiguousarray(self.pos, dtype=np.float64).reshape(-1, 3)
        self.ids = np.ascontiguousarray(self.ids, dtype=np.int64).reshape(-1)
        if len(self.pos) != len(self.ids):
            raise ValidationError(
                f"positions ({len(self.pos)}) and ids ({len(self.ids)}) length mismatch")

    def __len__(self):
        return len(self.ids)

    def center(self) -> np.ndarray:
        """Translate to the geometric centre; returns the old centre
        (src/structure.rs:197-207)."""
        if len(self.pos) == 0:
            return np.zeros(3)
        c = self.pos.mean(axis=0)
        self.pos = self.pos - c
        return c

    def set_positions(self, pos_angstrom: np.ndarray) -> None:
        """Replace the coordinates with a frame of the same atom count
        (src/structure.rs:220-232; frames here are already in Å)."""
        pos = np.asarray(pos_angstrom, dtype=np.float64).reshape(-1, 3)
        if len(pos) != len(self.pos):
            raise ValidationError(
                f"number of atoms in structure ({len(self.pos)}) does not match "
                f"trajectory frame ({len(pos)})")
        self.pos = np.ascontiguousarray(pos)


def parse_xyz(text: str) -> List[Tuple[str, Tuple[float, float, float]]]:
    """Lenient XYZ (src/input.rs:143-170): blank, ';' and '#' lines and lines
    that do not parse as ``name x y z`` are skipped."""
    atoms = []
    for line in text.splitlines():
        t = line.strip()
        if not t or t.startswith(";") or t.startswith("#"):
            continue
        parts = t.split()
        if len(parts) < 4:
            continue
        try:
            x, y, z = float(parts[1]), float(parts[2]), float(parts[3])
        except ValueError:
            continue
        atoms.append((parts[0], (x, y, z)))
    return atoms


def structure_from_xyz(path_or_text, formfactors: FormFactorMap, *, is_text: bool = False) -> Structure:
    """Read an XYZ file and resolve atom names to species ids by name."""
    text = path_or_text if is_text else open(path_or_text, "r", encoding="utf-8").read()
    atoms = parse_xyz(text)
    if not atoms:
        raise ValidationError("no atoms found in XYZ input")
    names = {k.name: i for i, k in enumerate(formfactors.kinds())}
    ids = []
    for name, _ in atoms:
        if name not in names:
            raise ValidationError(f"unknown atom kind '{name}'")
        ids.append(names[name])
    return Structure(np.array([p for _, p in atoms]), np.array(ids))
