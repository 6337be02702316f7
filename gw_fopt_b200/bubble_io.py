"""Bubble CSV files, as the reference's LatticeBubbles reads and writes them
(rust/bubble-gw/src/many_bubbles/lattice_bubbles.rs:480-572): one bubble per
row, four columns t, x, y, z, an optional header row "t,x,y,z", every row the
same length.  Host utilities beside the drop-in surface (the reference exposes
them in Rust only).
"""
from __future__ import annotations

import csv

import numpy as np

from .many_bubbles import LatticeBubbles


def load_bubbles_from_csv(path, has_headers=False):
    """(n, 4) float64 [t, x, y, z] (LB:510-528): a header row is skipped when has_headers;
    rows of unequal length or a column count other than 4 raise ValueError."""
    with open(path, newline="") as f:
        rows = list(csv.reader(f))
    if has_headers and rows:
        rows = rows[1:]
    rows = [r for r in rows if r]
    if not rows:
        return np.zeros((0, 4))
    n = len(rows[0])
    if any(len(r) != n for r in rows):
        raise ValueError(f"CSV error: found records with different lengths in {path}")
    if n != 4:
        raise ValueError("Invalid number of columns: expected 4 [t, x, y, z]")
    return np.array([[float(v) for v in r] for r in rows], dtype=np.float64)


def write_bubbles_to_csv(bubbles, path, has_headers=False):
    """Writes (n, 4) bubbles (LB:530-543); values in shortest round-trip form."""
    b = np.asarray(bubbles, dtype=np.float64)
    if b.ndim != 2 or b.shape[1] != 4:
        raise ValueError("Invalid number of columns: expected 4 [t, x, y, z]")
    with open(path, "w", newline="") as f:
        wr = csv.writer(f, lineterminator="\n")
        if has_headers:
            wr.writerow(["t", "x", "y", "z"])
        for row in b:
            wr.writerow([repr(float(v)) for v in row])


def from_csv_files(interior_path, exterior_path, lattice, has_headers=False):
    """LatticeBubbles from two CSV files (LB:488-498), validated as LatticeBubbles(...) is."""
    return LatticeBubbles(lattice, load_bubbles_from_csv(interior_path, has_headers),
                          load_bubbles_from_csv(exterior_path, has_headers))


def save_to_csv_files(lattice_bubbles, interior_path, exterior_path, has_headers=False):
    """Writes the interior and exterior bubbles of a LatticeBubbles (LB:545-571)."""
    write_bubbles_to_csv(lattice_bubbles.bubbles_interior, interior_path, has_headers)
    write_bubbles_to_csv(lattice_bubbles.bubbles_exterior, exterior_path, has_headers)
