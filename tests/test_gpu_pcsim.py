"""The phase-contrast data simulator on the GPU (through the C ABI) against the
reference's own outputs.

Fixture: tests/golden/pcsim_reference.npz (the reference's
phcontomo_forward_project built from source; tests/golden/gen_golden_pcsim.py).
Tolerances:
* projections SimMagProjs / SimPhaseProjs: 1e-12 relative to the largest
  value (FP64 on both sides; only the summation order differs);
* measurements: 2e-5 relative per pixel (the GPU's Fresnel transform is FP32,
  the reference's FP64); the noise draws are the reference's own sequence, so a
  different draw would differ by ~sqrt(m) ~ 2 % and fail;
* at the full default phantom size (512 x 512 x 128, 180 views, a 128 x 256
  detector) a zero phantom leaves |2500 + 50 n| per pixel: every one of the
  5.9 M noise values is checked against the oracle's randlib normal()
  sequence to 1e-6 relative.
"""
import os

import numpy as np
import pytest

import pcmbir_oracle as P
from phasecon_b200 import pcmbir as PC

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "pcsim_reference.npz"))
CASES = sorted({k.split("_")[0] for k in GOLD.files})


def params(c):
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = GOLD[f"{c}_params"]
    return int(P_xy), int(P_z), int(rows), int(cols), int(V), float(vox), float(rot), float(dist), float(en), float(dob)


@pytest.mark.parametrize("c", CASES)
def test_simulator_matches_reference(c):
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = params(c)
    o = PC.sim_options(phantom_xy=P_xy, phantom_z=P_z, write_files=0)
    meas, br, avg, pm, pp = PC.simulate(GOLD[f"{c}_mag"], GOLD[f"{c}_phase"], GOLD[f"{c}_angles"], rows, cols, vox,
                                        rot, dist, en, options=o, projections=True)
    for got, ref in ((pm, GOLD[f"{c}_projs_mag"]), (pp, GOLD[f"{c}_projs_phase"])):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    ref = GOLD[f"{c}_meas"]
    assert np.abs(meas / ref - 1).max() < 2e-5
    np.testing.assert_array_equal(br, GOLD[f"{c}_brights"])
    assert avg == pytest.approx(float(GOLD[f"{c}_avg"]), rel=2e-5)


def test_simulator_matches_oracle_at_a_larger_size():
    """128 x 128 x 32 phantom, 40 views, 32 x 64 detector against the oracle
    restatement (itself pinned to the reference): the same tolerances."""
    rng = np.random.default_rng(7)
    P_xy, P_z, rows, cols, V = 128, 32, 16, 64, 40
    z, y, x = np.meshgrid(np.arange(P_z) + 0.5, np.arange(P_xy) + 0.5, np.arange(P_xy) + 0.5, indexing="ij")
    mag = np.zeros((P_z, P_xy, P_xy), np.float32)
    ph = np.zeros_like(mag)
    for _ in range(6):
        c = rng.uniform([0.3 * P_z, 0.3 * P_xy, 0.3 * P_xy], [0.7 * P_z, 0.7 * P_xy, 0.7 * P_xy])
        r = rng.uniform(0.05, 0.15) * P_xy
        inside = (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 < r * r
        d = rng.uniform(1e-7, 3e-7)
        ph[inside] += d
        mag[inside] += d / 100
    ang = np.sort(rng.uniform(0, np.pi, V)).astype(np.float32)
    o = PC.sim_options(phantom_xy=P_xy, phantom_z=P_z, write_files=0)
    meas, br, avg, pm, pp = PC.simulate(mag, ph, ang, rows, cols, 1.0, 31.0, 5e4, 20.0, options=o, projections=True)
    ref_meas, ref_pm, ref_pp = P.simulate(mag, ph, ang, rows, cols, 1.0, 31.0, 5e4, 20.0)
    for got, ref in ((pm, ref_pm), (pp, ref_pp)):
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(meas / ref_meas - 1).max() < 2e-5


def test_dropin_reads_phantoms_and_writes_reference_files(tmp_path):
    c = CASES[0]
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = params(c)
    GOLD[f"{c}_mag"].tofile(tmp_path / "mag_in.bin")
    GOLD[f"{c}_phase"].tofile(tmp_path / "phase_in.bin")
    saved = PC.sim_options()
    try:
        PC.set_sim_options(PC.sim_options(phantom_xy=P_xy, phantom_z=P_z, write_files=1,
                                          mag_phantom_path=str(tmp_path / "mag_in.bin"),
                                          phase_phantom_path=str(tmp_path / "phase_in.bin")))
        meas = np.zeros((V, rows, cols), np.float32)
        br = np.zeros((rows, cols), np.float32)
        PC.phcontomo_forward_project(meas, br, GOLD[f"{c}_angles"], rows, cols, V, vox, rot, dist, en, dob,
                                     workdir=str(tmp_path))
    finally:
        PC.set_sim_options(saved)
    assert np.abs(meas / GOLD[f"{c}_meas"] - 1).max() < 2e-5
    assert np.all(br == 2500.0)
    n = V * P_z * P_xy
    for name, ref in (("SimMagProjs", GOLD[f"{c}_projs_mag"]), ("SimPhaseProjs", GOLD[f"{c}_projs_phase"])):
        got = np.fromfile(tmp_path / f"{name}.bin", np.float64)
        assert got.size == n
        assert np.abs(got.reshape(ref.shape) - ref).max() <= 1e-12 * np.abs(ref).max()
    for name, ph in (("mag_phantom", GOLD[f"{c}_mag"]), ("phase_phantom", GOLD[f"{c}_phase"])):
        np.testing.assert_array_equal(np.fromfile(tmp_path / f"{name}.bin", np.float64), ph.astype(np.float64).ravel())


def test_noise_sequence_at_the_full_default_size():
    o = PC.sim_options(write_files=0)
    assert (o.phantom_xy, o.phantom_z) == (512, 128)
    V, rows, cols = 180, 128, 256
    z = np.zeros((128, 512, 512), np.float32)
    ang = np.linspace(0, np.pi, V, endpoint=False).astype(np.float32)
    meas, br, avg = PC.simulate(z, z, ang, rows, cols, 1.0, 128.0, 5e4, 20.0, options=o)
    n = P.randlib_normals(meas.size).reshape(meas.shape)
    ref = np.abs(2500.0 + 50.0 * n).astype(np.float32)
    assert np.abs(meas / ref - 1).max() < 1e-6
