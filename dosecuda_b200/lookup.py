"""Beam-model lookup-table readers.

The table formats are the reference's, unchanged (DoseCUDA/lookuptables/**,
read by plan_impt.py:17-103 and plan_imrt.py:192-271).  The shipped tables
live in ``dosecuda_b200/lookuptables`` (copied from the reference with its
GPL-2.0 licence); ``DOSECUDA_LOOKUPTABLES`` points elsewhere.
"""
from __future__ import annotations

import os

import numpy as np
import pandas as pd

_DEFAULT_ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lookuptables")

LUT_ROWS = 400  # depth rows per energy the proton engine uses (plan_impt.py:73-80)


def table_root() -> str:
    return os.environ.get("DOSECUDA_LOOKUPTABLES", _DEFAULT_ROOT)


def table_path(*parts: str) -> str:
    return os.path.join(table_root(), *parts)


def read_key_values(path: str) -> dict:
    """``key, v1, v2, ...`` lines -> {key: [str values]} (machine_geometry.csv,
    beam_parameters.csv)."""
    out = {}
    with open(path, "r") as f:
        for line in f:
            parts = line.rstrip("\n").split(",")
            if len(parts) >= 2 and parts[0].strip():
                out[parts[0].strip()] = parts[1:]
    return out


def read_proton_energy(path: str):
    """One ``energy_NNN.csv``: line 2 holds energy, R80, A, B, C; from line 5 on
    ``depth,sigma,idd`` rows, of which the first LUT_ROWS are used."""
    with open(path, "r") as f:
        f.readline()
        params = [float(p) for p in f.readline().split(",")]
        f.readline()
        f.readline()
        rows = []
        for line in f:
            if len(rows) >= LUT_ROWS:
                break
            p = line.split(",")
            rows.append((float(p[0]), float(p[1]), float(p[2])))
    return params, rows
