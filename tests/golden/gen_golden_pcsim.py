"""Golden fixtures for the phase-contrast data simulator, from the reference itself.

    python tests/golden/gen_golden_pcsim.py

Runs the reference's phcontomo_forward_project (PCMBIR_3D/XT_Engine.c:199-253,
XT_genSinogram.c:59-343), built from source with the FP64 FFTW-API shim and
the phantom sizes / paths made settable (oracle/Makefile target ``ref_pc``), on
seeded sphere phantoms, and writes tests/golden/pcsim_reference.npz: for each
case the inputs, the measurements, the FP64 projections SimMagProjs /
SimPhaseProjs and the average of the measurements.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402

# (P_xy, P_z, proj_rows, proj_cols, proj_num, vox_wid, rot_center)
CASES = [(32, 8, 4, 16, 6, 2.0, 8.0), (16, 8, 8, 16, 5, 1.0, 7.5)]


def spheres(P_xy, P_z, rng, n=4):
    """Absorption (beta-like) and refractive-index-decrement (delta-like)
    phantoms of n random spheres, in phantom voxels."""
    z, y, x = np.meshgrid(np.arange(P_z) + 0.5, np.arange(P_xy) + 0.5, np.arange(P_xy) + 0.5, indexing="ij")
    mag = np.zeros((P_z, P_xy, P_xy))
    ph = np.zeros((P_z, P_xy, P_xy))
    for _ in range(n):
        c = rng.uniform([0.3 * P_z, 0.25 * P_xy, 0.25 * P_xy], [0.7 * P_z, 0.75 * P_xy, 0.75 * P_xy])
        r = rng.uniform(0.15, 0.3) * P_xy
        inside = (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 < r * r
        d = rng.uniform(1e-7, 5e-7)
        ph[inside] += d
        mag[inside] += d / 100
    return mag.astype(np.float32), ph.astype(np.float32)


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref_pc"], check=True)
    out = {}
    for k, (P_xy, P_z, rows, cols, V, vox, rot) in enumerate(CASES):
        rng = np.random.default_rng(100 + k)
        mag, ph = spheres(P_xy, P_z, rng)
        angles = np.sort(rng.uniform(0, np.pi, V)).astype(np.float32)
        dist, energy, dob = 5e4, 20.0, 100.0
        with tempfile.TemporaryDirectory() as td:
            meas, br, pm, pp, _, _ = O.ref_pc_forward_project(mag, ph, angles, rows, cols, vox, rot, dist, energy,
                                                              dob, td)
        out[f"c{k}_params"] = np.array([P_xy, P_z, rows, cols, V, vox, rot, dist, energy, dob])
        out[f"c{k}_mag"] = mag
        out[f"c{k}_phase"] = ph
        out[f"c{k}_angles"] = angles
        out[f"c{k}_meas"] = meas
        out[f"c{k}_brights"] = br
        out[f"c{k}_projs_mag"] = pm
        out[f"c{k}_projs_phase"] = pp
        out[f"c{k}_avg"] = np.float64(meas.astype(np.float64).mean())
    np.savez_compressed(os.path.join(HERE, "pcsim_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "pcsim_reference.npz"))


if __name__ == "__main__":
    main()
