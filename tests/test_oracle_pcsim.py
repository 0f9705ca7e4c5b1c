"""The data simulator's oracle pinned against the reference (CPU only), and the
drop-in's argument checks.

Fixture: tests/golden/pcsim_reference.npz, outputs of the reference's own
phcontomo_forward_project (PCMBIR_3D/XT_Engine.c:199-253) built from source
(tests/golden/gen_golden_pcsim.py). From the reference's FP64 projections, the
oracle's field, windowed Fresnel transform, detector averaging and randlib
normal() noise reproduce the reference's measurements bit for bit.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
import pcmbir_oracle as P

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "pcsim_reference.npz"))
CASES = sorted({k.split("_")[0] for k in GOLD.files})


def params(c):
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = GOLD[f"{c}_params"]
    return int(P_xy), int(P_z), int(rows), int(cols), int(V), float(vox), float(rot), float(dist), float(en), float(dob)


@pytest.mark.parametrize("c", CASES)
def test_oracle_measurements_match_reference_bit_exact(c):
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = params(c)
    g = P.sim_geometry(P_xy, P_z, rows, cols, vox, en, dist)
    m = P.sim_from_projections(GOLD[f"{c}_projs_mag"], GOLD[f"{c}_projs_phase"], g, rows, cols)
    np.testing.assert_array_equal(m, GOLD[f"{c}_meas"])
    assert np.all(GOLD[f"{c}_brights"] == 2500.0)


@pytest.mark.parametrize("c", CASES)
def test_oracle_projections_match_reference(c):
    """Projections to 1e-13 of the largest value (FP64, other summation order)."""
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = params(c)
    meas, pm, pp = P.simulate(GOLD[f"{c}_mag"], GOLD[f"{c}_phase"], GOLD[f"{c}_angles"], rows, cols, vox, rot, dist, en)
    for got, ref in ((pm, GOLD[f"{c}_projs_mag"]), (pp, GOLD[f"{c}_projs_phase"])):
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.abs(meas / GOLD[f"{c}_meas"] - 1).max() < 1e-6


def test_random2_states_known_answers():
    """randlib's published first values from seed 1 (PCMBIR_3D/randlib.c:69-90)."""
    s = P.random2_states(1, 5)
    assert list(s) == [16807, 282475249, 1622650073, 984943658, 1144108930]
    # block skip-ahead agrees with the one-by-one recurrence across block edges
    x, ref = 761521, []
    for _ in range(9000):
        x = x * 16807 % 2147483647
        ref.append(x)
    np.testing.assert_array_equal(P.random2_states(761521, 9000), np.array(ref, np.uint64))


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
def test_random2_states_match_the_reference_generator():
    np.testing.assert_array_equal(P.random2_states(761521, 1000).astype(np.float64) / P.PM_MODULUS,
                                  O.ref_random2_sequence(761521, 1000))


@pytest.mark.skipif(not O.ref_pc_available(), reason="reference build absent")
def test_live_reference_reproduces_fixture():
    c = CASES[0]
    P_xy, P_z, rows, cols, V, vox, rot, dist, en, dob = params(c)
    with tempfile.TemporaryDirectory() as td:
        meas, br, pm, pp, mg, ph = O.ref_pc_forward_project(GOLD[f"{c}_mag"], GOLD[f"{c}_phase"],
                                                            GOLD[f"{c}_angles"], rows, cols, vox, rot, dist, en,
                                                            dob, td)
    np.testing.assert_array_equal(meas, GOLD[f"{c}_meas"])
    np.testing.assert_array_equal(pm, GOLD[f"{c}_projs_mag"])
    np.testing.assert_array_equal(mg, GOLD[f"{c}_mag"].astype(np.float64))


def test_dropin_rejects_what_the_reference_rejects(tmp_path):
    """Argument checks of XT_Engine.c:214-217 and a missing phantom file return -1
    (no GPU work happens before them)."""
    from phasecon_b200 import MbirError
    from phasecon_b200 import pcmbir as PC
    saved = PC.sim_options()
    try:
        PC.set_sim_options(PC.sim_options(phantom_xy=32, phantom_z=8,
                                          mag_phantom_path=str(tmp_path / "missing_mag.bin"),
                                          phase_phantom_path=str(tmp_path / "missing_phase.bin")))
        ang = np.zeros(3, np.float32)
        for rows, cols in [(2, 16), (4, 15)]:  # fewer than 4 rows, odd column count
            m = np.zeros((3, rows, cols), np.float32)
            b = np.zeros((rows, cols), np.float32)
            with pytest.raises(MbirError):
                PC.phcontomo_forward_project(m, b, ang, rows, cols, 3, 1.0, 8.0, 5e4, 20.0, 100.0)
        m = np.zeros((3, 4, 16), np.float32)
        b = np.zeros((4, 16), np.float32)
        with pytest.raises(MbirError, match="Error in reading file"):
            PC.phcontomo_forward_project(m, b, ang, 4, 16, 3, 1.0, 8.0, 5e4, 20.0, 100.0)
        with pytest.raises(MbirError, match="finer than the phantom"):
            PC.phcontomo_forward_project(np.zeros((3, 16, 64), np.float32), np.zeros((16, 64), np.float32), ang,
                                         16, 64, 3, 1.0, 8.0, 5e4, 20.0, 100.0)
    finally:
        PC.set_sim_options(saved)
