"""The oracle restatement pinned against the reference's own outputs (CPU only).

Golden fixtures (tests/golden/mbir4d_reference.npz) are outputs of the
reference C built from source, made by tests/golden/gen_golden.py; where the
reference build itself is present (oracle/_ref/libref_mbir4d.so) a few checks
also run against it live.
"""
import os

import numpy as np
import pytest

import oracle as O
from phasecon_b200 import phantoms as P

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "mbir4d_reference.npz"))


def golden_problem(prefix: str) -> O.Problem:
    s = GOLD[f"{prefix}_scalars"]
    return O.Problem(GOLD[f"{prefix}_projections"], GOLD[f"{prefix}_weights"], GOLD[f"{prefix}_proj_angles"],
                     GOLD[f"{prefix}_proj_times"], GOLD[f"{prefix}_recon_times"], int(s[0]), int(s[1]), int(s[2]),
                     int(s[3]), float(s[4]), float(s[5]), float(s[6]), float(s[7]), float(s[8]), float(s[9]),
                     quad_convex=int(s[10]), huber_delta=float(s[11]), huber_T=float(s[12]), mrf_p=float(s[13]))


def test_random2_matches_randlib_known_answer_table():
    # randlib.c:69-92 lists the first 20 outputs of random2() from seed 1
    seq = np.rint(O.random2_sequence(1, 20) * 2147483647).astype(np.int64)
    assert np.array_equal(seq, GOLD["randlib_seed1"])


def test_geometry_and_detector_response_bit_exact():
    pb = golden_problem("quad")
    orc = O.Oracle(pb)
    g = orc.g
    mine = [g.delta_r, g.delta_t, g.R0, g.RMax, g.T0, g.TMax, g.x0, g.y0, g.z0, g.delta_xy, g.delta_z, g.OffsetR,
            g.OffsetT, g.delta_recon, g.radius_obj, g.z_overlap, g.sigma_s_q, g.sigma_s_q_p, g.sigma_t_q,
            g.sigma_t_q_p, g.time_filter, g.N_z]
    assert np.array_equal(np.array(mine), GOLD["quad_geom_scalars"][:22])
    assert np.array_equal(np.array(g.spatial_filter[:]), GOLD["quad_filter"])
    assert np.array_equal(orc.H_r, GOLD["quad_H_r"])


@pytest.mark.parametrize("m", [1, 2])
def test_amatrix_columns_bit_exact(m):
    pb = golden_problem("amat")
    orc = O.Oracle(pb, mult_xy=m, mult_z=m)
    cnt, idx, val = GOLD[f"amat{m}_count"], GOLD[f"amat{m}_index"], GOLD[f"amat{m}_value"]
    n = pb.proj_cols // m
    for v in range(pb.proj_num):
        for j in range(n):
            for k in range(n):
                i2, v2 = orc.amatrix_column(v, j, k)
                c = cnt[v, j, k]
                assert len(i2) == c
                assert np.array_equal(i2, idx[v, j, k, :c])
                assert np.array_equal(v2, val[v, j, k, :c])
                if c:  # channels are contiguous (the CUDA table relies on it)
                    assert np.array_equal(i2, np.arange(i2[0], i2[0] + c))


def test_error_sinogram_and_cost():
    pb = golden_problem("quad")
    orc = O.Oracle(pb)
    obj = GOLD["quad_true_object"]
    e = orc.error_sino(obj)
    ref = GOLD["quad_err_at_true"]
    # the reference accumulates A x in float, the restatement in double
    assert np.abs(e - ref).max() <= 1e-5 * np.abs(ref).max()
    c, _, _ = orc.cost(ref, obj)
    assert c == pytest.approx(float(GOLD["quad_cost_at_true"]), rel=1e-12)


def test_huber_cost_and_selection():
    pb = golden_problem("huber")
    orc = O.Oracle(pb)
    obj = GOLD["huber_half_object"]
    ref = GOLD["huber_err"]
    sel = (np.abs(ref.astype(np.float64) * np.sqrt(orc.w.astype(np.float64))) < orc.g.huber_T).astype(np.uint8)
    assert np.array_equal(sel, GOLD["huber_select"])
    assert sel.min() == 0  # the branch is exercised
    c, _, _ = orc.cost(ref, obj)
    assert c == pytest.approx(float(GOLD["huber_cost"]), rel=1e-12)


def test_functional_substitution_bit_exact():
    pb = golden_problem("quad")
    orc = O.Oracle(pb)
    out = np.array([orc.functional_substitution(GOLD["fs_V"][i], GOLD["fs_th1"][i], GOLD["fs_th2"][i],
                                                GOLD["fs_nh"][i], GOLD["fs_nf"][i], GOLD["fs_tn"][i],
                                                GOLD["fs_tf"][i]) for i in range(len(GOLD["fs_V"]))])
    assert np.array_equal(out, GOLD["fs_out"])


def test_sequential_icd_reaches_reference_cost():
    """The restated voxel update, run as plain sequential ICD, converges to the
    reference's cost (its update order and NH-ICD schedule differ)."""
    pb = golden_problem("quad")
    orc = O.Oracle(pb)
    x = np.zeros(orc.shape, np.float32)
    e = orc.error_sino(x)
    c0 = orc.cost(e, x)[0]
    assert c0 == pytest.approx(GOLD["quad_icd20_cost"][0], rel=1e-9)
    rng = np.random.default_rng(0)
    n = orc.g.N_time * orc.g.N_y * orc.g.N_x
    last = c0
    for it in range(1, 31):
        orc.icd_pass(x, e, rng.permutation(n).astype(np.int32), it)
        c = orc.cost(e, x)[0]
        assert c <= last * (1 + 1e-9)
        last = c
    ref_final = GOLD["quad_icd20_cost"][-1]
    assert abs(last - ref_final) / ref_final < 1e-3
    drift = np.abs(orc.error_sino(x) - e).max()
    assert drift < 1e-4


def test_view_schedules_match_example_sidecars():
    a, t = P.interlaced_views(8, 256, 1024)
    assert np.array_equal(a, GOLD["example_cahn_proj_angles"])
    assert np.array_equal(t, GOLD["example_cahn_proj_times"])
    a, _, _ = P.uniform_views(256)
    assert np.array_equal(a, GOLD["example_shepp_proj_angles"])


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_live_reference_matches_fixture():
    pb = golden_problem("quad")
    geo = O.ref_geometry(pb)
    assert np.array_equal(geo["H_r"], GOLD["quad_H_r"])
    assert np.array_equal(O.ref_random2_sequence(1, 20) * 2147483647, GOLD["randlib_seed1"].astype(np.float64))


NH_GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "nhicd_reference.npz"))


def test_vsc_selection_matches_reference_fixture():
    """NH-ICD voxel-line selection (XT_NHICD.c:164-216): dense, sparse (ties at
    zero) and quantised (ties) magnitude maps, square and non-square."""
    for i in range(int(NH_GOLD["n"])):
        got = O.vsc_select(NH_GOLD[f"mag{i}"], int(NH_GOLD[f"lines{i}"]))
        assert np.array_equal(got, NH_GOLD[f"sel{i}"].astype(bool)), i


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_live_reference_vsc_selection():
    rng = np.random.default_rng(9)
    m = rng.exponential(1.0, (48, 48)).astype(np.float32)
    assert np.array_equal(O.vsc_select(m, 1500), O.ref_vsc_select(m, 1500))
