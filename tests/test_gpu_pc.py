"""Parity of the sm_100a phase-contrast path (through the C ABI) with the oracle and the reference.

Tolerances (stated per result; the GPU computes in FP32 with FP64 per-view sums):
* Fresnel / Hermitian transforms: max |diff| <= 2e-5 x max |ref| (FP32 FFT);
* Paganin retrieval: 1e-4 relative to max |ref|;
* one steepest-descent step: w within 1e-4, Omega within 1e-3 relative to the
  largest magnitude, the stopping statistic within 1e-3 relative;
* Nelder-Mead proximal sweep (the reference's raster order, and the optional
  colour-class order with the oracle run in the same order): the reference's
  stop rule is a 0.005 % relative vertex movement, so FP32 and FP64 searches
  that branch differently (the GPU's cost uses hardware log2 / exp2 and a fast
  division) stop at different points of a final simplex of about that
  relative size: median |diff| <= 3e-4 and max |diff| <= 1e-2 relative to
  max |z|;
* three ADMM iterations: cost history within 2e-3 relative, z within 5e-3.
"""
import os

import numpy as np
import pytest

import oracle as O
import pcmbir_oracle as P
from phasecon_b200.pcmbir import PcProblem, PcSession, default_options, phcontomo_reconstruct
from test_oracle_pc import GOLD, geom as gold_geom

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def scan(V, R, C, seed, energy=20.0, distance=5e4, dob=100.0, sig=0.05):
    """Seeded synthetic scan: smooth exit waves, random bright field, noisy
    amplitudes. Returns (PcProblem, PcGeom, y [V][R][C], D [R][C], z true)."""
    rng = np.random.default_rng(seed)
    g = P.PcGeom(rows=R, cols=C, energy_kev=energy, distance=distance, mag_sig_s=sig, phase_sig_s=sig,
                 delta_over_beta=dob)
    bright = (0.8 + 0.4 * rng.random((C, R))).astype(np.float32)          # [proj_rows][proj_cols]
    bavg = np.sqrt(np.mean(bright.astype(np.float64)))
    D = (np.sqrt(bright.astype(np.float64)) / bavg).T                    # [R][C]
    jj, kk = np.meshgrid(np.arange(R), np.arange(C), indexing="ij")
    meas = np.zeros((V, C, R), np.float32)
    zt = []
    for v in range(V):
        cj, ck = R * (0.3 + 0.4 * rng.random()), C * (0.3 + 0.4 * rng.random())
        zr = 0.02 + 0.03 * np.exp(-((jj - cj) ** 2 + (kk - ck) ** 2) / (0.05 * R * C))
        zi = zr * dob * 0.04
        w = np.exp(-zr) * (np.cos(-zi) + 1j * np.sin(-zi))
        amp = np.abs(P.fresnel(g, D * w)) + 0.002 * rng.normal(size=(R, C))
        meas[v] = ((amp * bavg) ** 2).T
        zt.append((zr, zi))
    y = np.sqrt(meas.astype(np.float64)).transpose(0, 2, 1) / bavg
    pb = PcProblem(measurements=meas, brights=bright, vox_wid=1.0, mag_sig_s=sig, mag_c_s=1.0, phase_sig_s=sig,
                   phase_c_s=1.0, obj2det_dist=distance, light_energy=energy, pag_regparam=dob)
    return pb, g, y, D, zt


def start_state(g, y, D, zt, seed):
    rng = np.random.default_rng(seed)
    zr0 = np.stack([z[0] * (1 + 0.1 * rng.normal(size=z[0].shape)) for z in zt])
    zi0 = np.stack([z[1] * (1 + 0.1 * rng.normal(size=z[1].shape)) for z in zt])
    zr0, zi0 = zr0.astype(np.float32).astype(np.float64), zi0.astype(np.float32).astype(np.float64)
    w0 = np.exp(-zr0) * (np.cos(-zi0) + 1j * np.sin(-zi0))
    w0 = w0.astype(np.complex64).astype(np.complex128)
    om0 = np.stack([P.phase_projection(g, y[v], D, w0[v]) for v in range(len(zt))]).astype(np.complex64)
    return zr0, zi0, w0, om0.astype(np.complex128)


def test_fresnel_transforms_match_reference_fixture():
    g = gold_geom()
    R, C = g.rows, g.cols
    pb = PcProblem(measurements=np.ones((1, C, R), np.float32), brights=np.ones((C, R), np.float32),
                   vox_wid=1.0, obj2det_dist=g.distance, light_energy=g.energy_kev)
    s = PcSession(pb)
    x = GOLD["fresnel_in"][None]
    assert rel(s.fresnel(x, herm=False)[0], GOLD["fresnel_fwd"]) < 2e-5
    assert rel(s.fresnel(x, herm=True)[0], GOLD["fresnel_herm"]) < 2e-5


@pytest.mark.parametrize("R,C", [(32, 16), (128, 64), (64, 256), (256, 256)])
def test_batched_fresnel_matches_oracle(R, C):
    V = 3
    pb, g, _, _, _ = scan(V, R, C, seed=R + C)
    s = PcSession(pb)
    rng = np.random.default_rng(7)
    x = rng.normal(size=(V, R, C)) + 1j * rng.normal(size=(V, R, C))
    x = x.astype(np.complex64).astype(np.complex128)
    for herm in (False, True):
        out = s.fresnel(x, herm)
        for v in range(V):
            assert rel(out[v], P.fresnel(g, x[v], herm)) < 2e-5, (R, C, herm, v)


def test_paganin_matches_reference_fixture():
    g = gold_geom()
    R, C = g.rows, g.cols
    y, D = GOLD["y"], np.abs(GOLD["D"])
    pb = PcProblem(measurements=(y ** 2).T[None].astype(np.float32), brights=(D ** 2).T.astype(np.float32),
                   vox_wid=1.0, obj2det_dist=g.distance, light_energy=g.energy_kev, pag_regparam=g.delta_over_beta)
    s = PcSession(pb)
    zr, zi = s.paganin()
    assert rel(zr[0], GOLD["pag_zr"]) < 1e-4
    assert rel(zi[0], GOLD["pag_zi"]) < 1e-4


def test_steepest_descent_step_matches_oracle():
    V, R, C = 3, 64, 32
    pb, g, y, D, zt = scan(V, R, C, seed=11)
    zr0, zi0, w0, om0 = start_state(g, y, D, zt, seed=12)
    buf = (w0 * (1.02 + 0.01j)).astype(np.complex64).astype(np.complex128)
    s = PcSession(pb)
    s.set_z(zr0, zi0)
    s.set_state(w=w0, v=np.zeros_like(w0), omega=om0)
    th = s.sd_step(buf)
    _, _, w1, _, om1 = s.get_state()
    for v in range(V):
        wr, omr, thr = P.sd_iter(g, y[v], om0[v], D, w0[v], np.ones((R, C)), buf[v])
        assert rel(w1[v], wr) < 1e-4, v
        assert rel(om1[v], omr) < 1e-3, v
        assert th[v] == pytest.approx(thr, rel=1e-3)


def nms_case(V, R, C, seed=21):
    pb, g, y, D, zt = scan(V, R, C, seed=seed)
    zr0, zi0, w0, om0 = start_state(g, y, D, zt, seed=seed + 1)
    rng = np.random.default_rng(seed + 2)
    vd = (0.01 * (rng.normal(size=w0.shape) + 1j * rng.normal(size=w0.shape))).astype(np.complex64)
    return pb, g, zr0, zi0, w0, om0, vd


def gpu_nms_sweep(pb, zr0, zi0, w0, om0, vd, **opts):
    s = PcSession(pb, default_options(**opts))
    s.set_z(zr0, zi0)
    s.set_state(w=w0, v=vd, omega=om0)
    s.nms_sweep()
    zr1, zi1, _, _, _ = s.get_state()
    s.close()
    return zr1, zi1


@pytest.mark.parametrize("order,lanes,ctas", [("raster", 1, 1), ("raster", 2, 1), ("raster", 4, 2), ("raster", 8, 4),
                                              ("raster", 8, 1), ("color", 1, 0), ("color", 4, 0), ("color", 8, 0)])
def test_nelder_mead_sweep_matches_oracle(order, lanes, ctas):
    """Every layout of the search (lanes per pixel, CTAs per view)."""
    V, R, C = 2, 32, 16
    pb, g, zr0, zi0, w0, om0, vd = nms_case(V, R, C)
    zr1, zi1 = gpu_nms_sweep(pb, zr0, zi0, w0, om0, vd, nms_order=0 if order == "raster" else 1, nms_lanes=lanes,
                             nms_ctas_per_view=ctas)
    for v in range(V):
        ar, ai = zr0[v].copy(), zi0[v].copy()
        P.nms_sweep(g, ar, ai, w0[v] - vd[v].astype(np.complex128), order=order)
        for got, ref in ((zr1[v], ar), (zi1[v], ai)):
            d = np.abs(got - ref) / np.abs(ref).max()
            assert np.median(d) <= 3e-4 and d.max() <= 1e-2, (v, float(np.median(d)), float(d.max()))


@pytest.mark.parametrize("lanes", [1, 4, 8])
def test_raster_sweep_does_not_depend_on_ctas_per_view(lanes):
    """The raster order is kept exactly however a view's anti-diagonals are
    dealt over the CTAs of its cluster: the same lanes per pixel give the same
    bits with 1, 2 or 4 CTAs per view (64 x 64 views: up to 32 pixels per
    anti-diagonal, so every CTA of a cluster has pixels)."""
    pb, g, zr0, zi0, w0, om0, vd = nms_case(3, 64, 64, seed=31)
    outs = [gpu_nms_sweep(pb, zr0, zi0, w0, om0, vd, nms_order=0, nms_lanes=lanes, nms_ctas_per_view=c)
            for c in (1, 2, 4)]
    for zr, zi in outs[1:]:
        assert np.array_equal(zr, outs[0][0]) and np.array_equal(zi, outs[0][1])


def test_phase_retrieval_admm_matches_oracle():
    V, R, C = 2, 32, 16
    pb, g, y, D, zt = scan(V, R, C, seed=31)
    zr0, zi0, w0, om0 = start_state(g, y, D, zt, seed=32)
    opt = default_options(pret_max_iter=3, sd_max_iter=10)
    s = PcSession(pb, opt)
    s.set_z(zr0, zi0)
    s.set_state(w=w0, omega=om0)
    costs, iters, st = s.run()
    zr1, zi1, w1, _, _ = s.get_state()
    assert list(iters) == [3] * V
    assert 0 < st.sd_steps <= V * 3 * 10
    for v in range(V):
        rz, ri, rw, _, _, rc = P.estimate_projection(g, y[v], om0[v], D, zr0[v], zi0[v], np.ones((R, C)), w0[v],
                                                      pret_iters=3, sd_iters=10)
        assert np.allclose(costs[v, :len(rc)], rc, rtol=2e-3), (v, costs[v], rc)
        assert rel(zr1[v], rz) < 5e-3 and rel(zi1[v], ri) < 5e-3
        assert rel(w1[v], rw) < 5e-3


def test_init_admm_matches_oracle():
    V, R, C = 2, 64, 64
    pb, g, y, D, zt = scan(V, R, C, seed=41)
    zr0, zi0, _, _ = start_state(g, y, D, zt, seed=42)
    s = PcSession(pb)
    s.set_z(zr0, zi0)
    s.init_admm()
    _, _, w, v, om = s.get_state()
    for k in range(V):
        wr = np.exp(-zr0[k]) * (np.cos(-zi0[k]) + 1j * np.sin(-zi0[k]))
        assert rel(w[k], wr) < 1e-6
        assert np.abs(v[k]).max() == 0
        assert rel(om[k], P.phase_projection(g, y[k], D, wr)) < 1e-3


def test_phcontomo_reconstruct_writes_reference_files(tmp_path):
    V, R, C = 2, 32, 16
    pb, g, y, D, zt = scan(V, R, C, seed=51)
    args = dict(measurements=pb.measurements, brights=pb.brights, proj_angles=np.zeros(V, np.float32),
                proj_times=np.arange(V, dtype=np.float32), recon_times=np.array([0, V], np.float32),
                proj_rows=C, proj_cols=R, proj_num=V, recon_num=1, vox_wid=1.0, rot_center=R / 2,
                mag_sig_s=pb.mag_sig_s, mag_sig_t=1.0, mag_c_s=1.0, mag_c_t=1.0, phase_sig_s=pb.phase_sig_s,
                phase_sig_t=1.0, phase_c_s=1.0, phase_c_t=1.0, convg_thresh=0.0, obj2det_dist=pb.obj2det_dist,
                light_energy=pb.light_energy, pag_regparam=pb.pag_regparam)
    phcontomo_reconstruct(**args, recon_type=1, workdir=str(tmp_path))
    pz = np.fromfile(tmp_path / "pag_mag_ret.bin", np.float64).reshape(V, R, C)
    zr, _ = PcSession(pb).paganin()
    assert np.array_equal(pz, zr.astype(np.float64))
    phcontomo_reconstruct(**args, recon_type=2, workdir=str(tmp_path))
    for name in ("mag_pret_aux", "phase_pret_aux", "omega_real", "omega_imag", "mag_pret_dual"):
        assert os.path.getsize(tmp_path / f"{name}.bin") == V * R * C * 8
    aux = np.fromfile(tmp_path / "mag_tomo_aux.bin", np.float64).reshape(V, R, C, 4)
    assert np.isfinite(aux).all()
    cost = np.fromfile(tmp_path / "pret_cost_proj_0.bin", np.float64)
    assert len(cost) >= 2 and cost[-1] < cost[0]


@pytest.mark.skipif(not O.ref_pc_available(), reason="reference build not present")
def test_phcontomo_reconstruct_matches_reference_files(tmp_path):
    """The drop-in phcontomo_reconstruct against the reference's own
    phcontomo_reconstruct (PCMBIR_3D/XT_Engine.c:82, built from source with the
    FP64 FFT shim) on the same seeded scan, recon_type 1 (Paganin) then 2 (the
    per-view phase-retrieval ADMM, 100 PRet iterations as shipped):
    * pag_mag_ret / pag_phase_ret: max |diff| <= 1e-4 x max |ref| (FP32 FFT);
    * pret_cost_proj_<i>: the same number of PRet iterations; the first five
      costs within 2e-3 relative (the three-iteration ADMM test's bound);
      over 100 iterations the FP32 and FP64 per-pixel searches (a nonconvex
      problem) drift apart, so at the end the GPU's cost must be no higher than
      the reference's by more than 1e-3 relative (it was 1 % lower when
      measured);
    * the final phase-retrieval state (mag/phase_pret_aux, omega_real/imag):
      RMSE within 5 % of the reference's dynamic range (the two end at nearby
      points of that drift)."""
    V, R, C = 2, 32, 16
    pb, g, y, D, zt = scan(V, R, C, seed=51)
    args = dict(measurements=pb.measurements, brights=pb.brights, proj_angles=np.zeros(V, np.float32),
                proj_times=np.arange(V, dtype=np.float32), recon_times=np.array([0, V], np.float32),
                proj_rows=C, proj_cols=R, proj_num=V, recon_num=1, vox_wid=1.0, rot_center=R / 2,
                mag_sig_s=pb.mag_sig_s, mag_sig_t=1.0, mag_c_s=1.0, mag_c_t=1.0, phase_sig_s=pb.phase_sig_s,
                phase_sig_t=1.0, phase_c_s=1.0, phase_c_t=1.0, convg_thresh=0.0, obj2det_dist=pb.obj2det_dist,
                light_energy=pb.light_energy, pag_regparam=pb.pag_regparam)
    gdir, rdir = tmp_path / "gpu", tmp_path / "ref"
    os.makedirs(gdir)
    for rt in (1, 2):
        phcontomo_reconstruct(**args, recon_type=rt, workdir=str(gdir))
        O.ref_pc_reconstruct(str(rdir), **args, recon_type=rt)

    def load(d, name):
        return np.fromfile(d / f"{name}.bin", np.float64)

    for name in ("pag_mag_ret", "pag_phase_ret"):
        assert rel(load(gdir, name), load(rdir, name)) < 1e-4, name
    for v in range(V):
        cg, cr = load(gdir, f"pret_cost_proj_{v}"), load(rdir, f"pret_cost_proj_{v}")
        assert len(cg) == len(cr), (v, len(cg), len(cr))
        assert np.allclose(cg[:5], cr[:5], rtol=2e-3, atol=0), (v, cg[:5], cr[:5])
        assert cg[-1] <= cr[-1] * (1 + 1e-3), (v, cg[-1], cr[-1])
    for name in ("mag_pret_aux", "phase_pret_aux", "omega_real", "omega_imag"):
        a, b = load(gdir, name), load(rdir, name)
        assert a.shape == b.shape, name
        assert np.sqrt(np.mean((a - b) ** 2)) <= 5e-2 * (b.max() - b.min()), name


def test_colour_class_sweep_reaches_the_raster_cost():
    """The Nelder-Mead proximal sweep in colour classes (four launches, no two
    8-neighbours in one class) against the reference's raster order (the
    wavefront kernel): the full per-view ADMM, 20 phase-retrieval iterations
    from the Paganin start on 6 views of 64 x 64. The colour-class order ends
    0.2-0.7 % above the raster order's phase-retrieval cost (measured), so it
    is not the default: the raster order is. Bound: within 1 %."""
    V, R, C = 6, 64, 64
    pb, g, y, D, zt = scan(V, R, C, seed=61)
    finals = []
    for order in (0, 1):
        s = PcSession(pb, default_options(pret_max_iter=20, nms_order=order))
        s.paganin()
        s.init_admm()
        costs, iters, _ = s.run()
        finals.append(np.array([c[np.isfinite(c)][-1] for c in costs]))
        s.close()
    raster, colour = finals
    assert np.all(np.abs(colour - raster) / np.abs(raster) < 1e-2), (raster, colour)


@pytest.mark.skipif(not O.ref_pc_available(), reason="reference build not present")
def test_one_phase_retrieval_iteration_at_the_phase_contrast_size_matches_reference(tmp_path):
    """One phase-retrieval iteration (Nelder-Mead sweep in the reference's
    raster order, steepest descent to its stop rule, dual update) of the
    phase-contrast scan at its full size -- 180 views of 256 x 256, every view
    batched on the GPU from the Paganin start -- against the reference's own
    estimate_complex_projection (PCMBIR_3D/XT_CmplxProjEst.c:91-229, built from
    source with the FP64 FFT shim) on four of the views from the same start.
    z comes out of the Nelder-Mead sweep, whose FP32 and FP64 searches stop at
    different points of a final simplex (the sweep's tolerance: median |diff|
    <= 3e-4 and max |diff| <= 1e-2 of the view's largest magnitude). w and
    Omega follow z through up to 100 steepest-descent steps whose FP32 and
    FP64 runs can stop a step apart: median |diff| <= 3e-4 and 99th
    percentile <= 1e-2 (measured: medians 2-4e-5, 99th percentiles 4-7e-3;
    0.2-0.6 % of the pixels differ by more than 1e-2, up to 0.17 for w and
    0.49 for Omega, at dark fringe pixels where y is a quarter to a half of
    its median). The phase-retrieval cost after the iteration within 1e-4
    relative (measured 4e-6 to 2e-5)."""
    from phasecon_b200 import workloads as W
    pb, _ = W.config_pc(seed=5)
    V, rows, cols = pb.dims
    R, C = cols, rows  # session layout [view][N_r][N_t] = [view][proj_cols][proj_rows]
    s = PcSession(pb, default_options(pret_max_iter=1, nms_order=0))
    s.paganin()
    s.init_admm()
    zr0, zi0, w0, _, om0 = s.get_state()
    costs, iters, _ = s.run()
    zr1, zi1, w1, _, om1 = s.get_state()
    s.close()
    assert list(set(iters.tolist())) == [1]
    g = P.PcGeom(rows=R, cols=C, energy_kev=pb.light_energy, distance=pb.obj2det_dist, mag_sig_s=pb.mag_sig_s,
                 phase_sig_s=pb.phase_sig_s, delta_over_beta=pb.pag_regparam)
    bavg = np.sqrt(np.mean(pb.brights.astype(np.float64)))
    D = (np.sqrt(pb.brights.astype(np.float64)) / bavg).T
    def stats(a, b):
        d = np.abs(np.asarray(a) - np.asarray(b)) / max(np.abs(b).max(), 1e-300)
        return float(np.median(d)), float(np.percentile(d, 99)), float(d.max())

    report = []
    for v in (0, 45, 90, 135):
        y = np.sqrt(pb.measurements[v].astype(np.float64)).T / bavg
        rz, ri, rw, _, rom, rc = O.ref_pc_estimate(g, y, om0[v], D, zr0[v], zi0[v], np.ones((R, C)), w0[v],
                                                    str(tmp_path / f"v{v}"), pret_iters=1)
        report.append({"view": v, "zr": stats(zr1[v], rz), "zi": stats(zi1[v], ri), "w": stats(w1[v], rw),
                       "omega": stats(om1[v], rom), "cost": abs(costs[v, 1] - rc[-1]) / abs(rc[-1])})
    print(report)
    for r in report:
        for k in ("zr", "zi"):
            med, _, mx = r[k]
            assert med <= 3e-4 and mx <= 1e-2, (r["view"], k, med, mx)
        for k in ("w", "omega"):
            med, p99, _ = r[k]
            assert med <= 3e-4 and p99 <= 1e-2, (r["view"], k, med, p99)
        assert r["cost"] < 1e-4, r
