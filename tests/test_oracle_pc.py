"""The phase-contrast oracle restatement pinned against the reference's outputs (CPU only).

Fixtures: tests/golden/pcmbir_reference.npz, outputs of the reference PCMBIR_3D
C built from source with the FP64 FFTW-API shim (tests/golden/gen_golden_pc.py).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
import pcmbir_oracle as P

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "pcmbir_reference.npz"))


def geom():
    s = GOLD["geom"]
    return P.PcGeom(rows=int(s[0]), cols=int(s[1]), delta_rows=s[2], delta_cols=s[3], energy_kev=s[4],
                    distance=s[5], mag_sig_s=s[6], mag_c_s=s[7], phase_sig_s=s[8], phase_c_s=s[9],
                    delta_over_beta=s[10], mrf_p=s[11])


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("herm", [False, True])
def test_fresnel_transforms(herm):
    g = geom()
    ref = GOLD["fresnel_herm" if herm else "fresnel_fwd"]
    assert rel(P.fresnel(g, GOLD["fresnel_in"], herm), ref) < 1e-13


def test_phase_projection_and_steepest_descent_step():
    g = geom()
    y, D, w0, lam = GOLD["y"], GOLD["D"], GOLD["w0"], GOLD["lam"]
    om0 = P.phase_projection(g, y, D, w0)
    assert rel(om0, GOLD["omega0"]) < 1e-12
    w1, om1, t = P.sd_iter(g, y, GOLD["omega0"], D, w0, lam, GOLD["sd_buf"])
    assert rel(w1, GOLD["sd_w1"]) < 1e-12
    assert rel(om1, GOLD["sd_omega1"]) < 1e-12
    assert t == pytest.approx(float(GOLD["sd_thresh"]), rel=1e-10)


def test_nelder_mead_bit_exact():
    g = geom()
    cf = P.NmsCost(g)
    for i in range(len(GOLD["nms_br"])):
        nr = GOLD["nms_nbr_r"][i].reshape(3, 3).tolist()
        ni = GOLD["nms_nbr_i"][i].reshape(3, 3).tolist()
        fl = GOLD["nms_flag"][i].reshape(3, 3).astype(bool).tolist()
        zr, zi, _ = P.nelder_mead(cf, nr[1][1], ni[1][1], GOLD["nms_br"][i], GOLD["nms_bi"][i], nr, ni, fl)
        assert zr == GOLD["nms_zr"][i] and zi == GOLD["nms_zi"][i]


def test_paganin():
    g = geom()
    zr, zi = P.paganin(g, GOLD["y"], GOLD["D"])
    assert rel(zr, GOLD["pag_zr"]) < 1e-12
    assert rel(zi, GOLD["pag_zi"]) < 1e-12


def test_phase_retrieval_admm_three_iterations():
    g = geom()
    zr, zi, w, v, om, costs = P.estimate_projection(g, GOLD["y"], GOLD["omega0"], GOLD["D"], GOLD["zr0"],
                                                    GOLD["zi0"], GOLD["lam"], GOLD["w0"], pret_iters=3, sd_iters=10)
    assert rel(zr, GOLD["est_zr"]) < 1e-10
    assert rel(zi, GOLD["est_zi"]) < 1e-10
    assert rel(w, GOLD["est_w"]) < 1e-10
    assert np.allclose(costs, GOLD["est_cost"], rtol=1e-10)


def test_fftw_shim_matches_numpy():
    """The FP64 FFTW-API shim the reference is built with agrees with numpy.fft."""
    if not O.ref_pc_available():
        pytest.skip("reference build not present")
    g = geom()
    x = GOLD["fresnel_in"]
    # a transfer-free check: the forward transform with distance -> tiny window effect is not
    # available through the harness, so compare the full Fresnel pipeline instead
    assert rel(O.ref_pc_fresnel(g, x, True), np.fft.ifft2(np.fft.fft2(x) * g.transfer(True))) < 1e-13
