"""Batch modules shipped with goss_b200 (generated sources, built in-tree).

Each entry lists the (shipped model variant, explicit solver) kinds that one
persistent kernel covers; ``python -m goss_b200.models.generate`` writes the
sources into ``goss_b200/batches/<name>/``.
"""
from __future__ import annotations

from pathlib import Path
from typing import Dict, List

HERE = Path(__file__).resolve().parent

FIELDS4 = ["g_Kr", "g_Ks", "g_CaL", "g_to"]

# name, kinds: (model name, field parameters, solver)
SHIPPED_BATCHES: List[Dict] = [
    dict(name="cardiac_mix", kinds=[
        ("fitzhughnagumo", ["a", "b"], "RK4"),
        ("oscilator", ["a", "b"], "RK4"),
        ("tentusscher_2004_mcell", FIELDS4, "GRL1"),
        ("tentusscher_panfilov_2006_M_cell", FIELDS4, "GRL1"),
    ]),
]


def batch_dirs() -> List[Path]:
    return sorted(p.parent for p in HERE.glob("*/batch.json"))
