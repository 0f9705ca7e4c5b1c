"""Golden fixtures for the phase-contrast (PCMBIR_3D) path, from the reference itself.

    python tests/golden/gen_golden_pc.py

Every output array here comes from the reference C (PCMBIR_3D) built from
source with the FP64 FFTW-API shim (oracle/Makefile target ``ref_pc``); the
inputs are seeded. Writes tests/golden/pcmbir_reference.npz.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
import pcmbir_oracle as P  # noqa: E402


def main():
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref_pc"], check=True)
    rng = np.random.default_rng(42)
    R, Cc = 32, 16
    g = P.PcGeom(rows=R, cols=Cc, delta_rows=1.0, delta_cols=1.0, mag_sig_s=0.05, phase_sig_s=0.05)
    out = {"geom": np.array([R, Cc, g.delta_rows, g.delta_cols, g.energy_kev, g.distance, g.mag_sig_s, g.mag_c_s,
                             g.phase_sig_s, g.phase_c_s, g.delta_over_beta, g.mrf_p])}
    x = rng.normal(size=(R, Cc)) + 1j * rng.normal(size=(R, Cc))
    out["fresnel_in"] = x
    out["fresnel_fwd"] = O.ref_pc_fresnel(g, x, False)
    out["fresnel_herm"] = O.ref_pc_fresnel(g, x, True)
    # a smooth synthetic exit wave and measurement
    jj, kk = np.meshgrid(np.arange(R), np.arange(Cc), indexing="ij")
    zr = 0.05 + 0.04 * np.exp(-((jj - R / 2) ** 2 + (kk - Cc / 2) ** 2) / 40.0)
    zi = zr * 4.0
    D = (0.9 + 0.1 * rng.random((R, Cc))) + 0j
    wt = np.exp(-zr) * (np.cos(-zi) + 1j * np.sin(-zi))
    y = np.abs(P.fresnel(g, D * wt)) + 0.005 * rng.normal(size=(R, Cc))
    zr0 = zr * (1 + 0.1 * rng.normal(size=(R, Cc)))
    zi0 = zi * (1 + 0.1 * rng.normal(size=(R, Cc)))
    w0 = np.exp(-zr0) * (np.cos(-zi0) + 1j * np.sin(-zi0))
    lam = np.ones((R, Cc))
    out.update(y=y, D=D, zr0=zr0, zi0=zi0, w0=w0, lam=lam)
    om0 = O.ref_pc_phase_projection(g, y, D, w0)
    out["omega0"] = om0
    buf = w0 * 1.02
    w1, om1, t1 = O.ref_pc_sd_iter(g, y, om0, D, w0, lam, buf)
    out.update(sd_buf=buf, sd_w1=w1, sd_omega1=om1, sd_thresh=np.float64(t1))
    n = 64
    br = rng.normal(0.9, 0.05, n)
    bi = rng.normal(-0.3, 0.05, n)
    nbr_r = 0.05 + 0.02 * rng.random((n, 9))
    nbr_i = 0.2 + 0.05 * rng.random((n, 9))
    fl = (rng.random((n, 9)) > 0.1).astype(np.uint8)
    rr, ri, its = O.ref_pc_nms(g, nbr_r[:, 4].copy(), nbr_i[:, 4].copy(), br, bi, nbr_r, nbr_i, fl)
    out.update(nms_br=br, nms_bi=bi, nms_nbr_r=nbr_r, nms_nbr_i=nbr_i, nms_flag=fl, nms_zr=rr, nms_zi=ri,
               nms_iters=its)
    pr, pi = O.ref_pc_paganin(g, y, D)
    out.update(pag_zr=pr, pag_zi=pi)
    er = O.ref_pc_estimate(g, y, om0, D, zr0, zi0, lam, w0, tempfile.mkdtemp(), pret_iters=3, sd_iters=10)
    out.update(est_zr=er[0], est_zi=er[1], est_w=er[2], est_v=er[3], est_omega=er[4], est_cost=er[5])
    np.savez_compressed(os.path.join(HERE, "pcmbir_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "pcmbir_reference.npz"))


if __name__ == "__main__":
    main()
