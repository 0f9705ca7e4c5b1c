"""Golden fixtures for the NH-ICD voxel-line selection, from the reference itself.

    python tests/golden/gen_golden_nhicd.py

Runs the reference's VSC_based_Voxel_Line_Select (MBIR_4D/XT_NHICD.c:164-216,
built from source by oracle/Makefile target ``ref``) on seeded update-magnitude
maps and writes tests/golden/nhicd_reference.npz.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402


def cases():
    rng = np.random.default_rng(2024)
    out = []
    for ny, nx in ((64, 64), (40, 56), (32, 32)):
        jj, kk = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        circle = (jj - ny / 2 + 0.5) ** 2 + (kk - nx / 2 + 0.5) ** 2 <= (min(ny, nx) / 2) ** 2
        dense = (rng.exponential(1e-3, (ny, nx)) * circle).astype(np.float32)
        sparse = (rng.exponential(1e-3, (ny, nx)) * (rng.random((ny, nx)) < 0.03) * circle).astype(np.float32)
        ties = (np.round(rng.random((ny, nx)) * 4) / 4 * circle).astype(np.float32)
        for m in (dense, sparse, ties):
            out.append((m, int(circle.sum())))
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    d = {}
    for i, (m, n_lines) in enumerate(cases()):
        d[f"mag{i}"] = m
        d[f"lines{i}"] = np.int32(n_lines)
        d[f"sel{i}"] = O.ref_vsc_select(m, n_lines).astype(np.uint8)
    d["n"] = np.int32(len(cases()))
    np.savez_compressed(os.path.join(HERE, "nhicd_reference.npz"), **d)
    print("wrote", os.path.join(HERE, "nhicd_reference.npz"))


if __name__ == "__main__":
    main()
