"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the phasecon sources (the reference C is built from
them by ``make -C oracle ref``):

    PHASECON_REFERENCE_ROOT=/path/to/phasecon python tests/golden/gen_golden.py

Every array saved here is an OUTPUT OF THE REFERENCE C code, built from source
with a single-rank MPI shim (oracle/Makefile), or a vector shipped with the
reference (the example sidecars, the random-number table in randlib.c's
comments). The fixtures pin the oracle restatement (tests/test_oracle.py) and
the CUDA path (tests/test_gpu_*.py) without needing the reference at run time.
"""
from __future__ import annotations

import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from problems import make_problem  # noqa: E402


def randlib_table(ref_root: str) -> np.ndarray:
    """The 20-number known-answer table in randlib.c's comment (seed 1)."""
    txt = open(os.path.join(ref_root, "Source_Code/MBIR_4D/randlib.c")).read()
    block = txt[txt.index("TABLE:"):]
    block = block[:block.index("*/")]
    nums = [int(x) for x in re.findall(r"^\s*(\d+)\s*$", block, re.M)]
    assert len(nums) == 20, nums
    return np.array(nums, np.int64)


def problem_arrays(pb) -> dict:
    return dict(projections=pb.projections, weights=pb.weights, proj_angles=pb.proj_angles,
                proj_times=pb.proj_times, recon_times=pb.recon_times,
                scalars=np.array([pb.proj_rows, pb.proj_cols, pb.proj_num, pb.recon_num, pb.vox_wid, pb.rot_center,
                                  pb.sig_s, pb.sig_t, pb.c_s, pb.c_t, pb.quad_convex, pb.huber_delta, pb.huber_T,
                                  pb.mrf_p], np.float64))


def main(ref_root: str) -> None:
    O.build(with_reference=True)
    out = {}

    # 1. a 2-frame problem with the quadratic data term
    pb, obj = make_problem(ncol=32, nrow=8, nview=40, nframe=2, seed=3, p=1.2, sig_t=0.02, moving=True)
    geo = O.ref_geometry(pb)
    err, sel, cost = O.ref_error_sino_and_cost(pb, obj)
    ref_obj, ref_cost, ref_updates = O.ref_reconstruct(pb, tempfile.mkdtemp(), max_iter=20, num_stages=1, threads=4)
    out.update({f"quad_{k}": v for k, v in problem_arrays(pb).items()})
    out.update(quad_true_object=obj, quad_H_r=geo["H_r"], quad_geom_scalars=geo["scal"], quad_filter=geo["filt"],
               quad_err_at_true=err, quad_cost_at_true=np.float64(cost), quad_icd20_cost=ref_cost,
               quad_icd20_object=ref_obj[:, 1:-1], quad_icd20_updates=np.int64(ref_updates))

    # 2. the generalised-Huber data term (quad_convex = 0), one frame, p = 1.1
    pbh, objh = make_problem(ncol=32, nrow=8, nview=36, nframe=1, seed=5, p=1.1, quad_convex=0,
                             huber_delta=0.2, huber_T=2.0)
    errh, selh, costh = O.ref_error_sino_and_cost(pbh, objh * 0.5)
    rh_obj, rh_cost, _ = O.ref_reconstruct(pbh, tempfile.mkdtemp(), max_iter=10, num_stages=1, threads=4)
    out.update({f"huber_{k}": v for k, v in problem_arrays(pbh).items()})
    out.update(huber_half_object=objh * 0.5, huber_err=errh, huber_select=selh, huber_cost=np.float64(costh),
               huber_icd10_cost=rh_cost, huber_icd10_object=rh_obj[:, 1:-1])

    # 3. A-matrix columns at 12 views (full scale and voxel scale 2)
    pba, _ = make_problem(ncol=32, nrow=8, nview=12, nframe=1, seed=1)
    for m in (1, 2):
        cnt, idx, val = O.ref_amatrix(pba, mult_xy=m, mult_z=m)
        out[f"amat{m}_count"], out[f"amat{m}_index"], out[f"amat{m}_value"] = cnt, idx, val
    out.update({f"amat_{k}": v for k, v in problem_arrays(pba).items()})

    # 4. surrogate solve samples
    rng = np.random.default_rng(11)
    n = 64
    V = rng.uniform(0, .02, n)
    th1 = rng.normal(0, 50, n)
    th2 = rng.uniform(10, 1e3, n)
    nh = rng.uniform(0, .02, (n, 27))
    nh[:, ::5] = V[:, None]
    nf = (rng.random((n, 27)) > 0.2).astype(np.uint8)
    tn = rng.uniform(0, .02, (n, 2))
    tf = (rng.random((n, 2)) > .3).astype(np.uint8)
    out.update(fs_V=V, fs_th1=th1, fs_th2=th2, fs_nh=nh, fs_nf=nf, fs_tn=tn, fs_tf=tf,
               fs_out=O.ref_functional_substitution(pb, V, th1, th2, nh, nf, tn, tf))

    # 5. vectors shipped with the reference
    out["randlib_seed1"] = randlib_table(ref_root)
    for ex in ("shepp-logan-3D", "cahn-hilliard-4D"):
        key = ex.split("-")[0]
        for f in ("proj_angles", "proj_times", "recon_times"):
            out[f"example_{key}_{f}"] = np.fromfile(os.path.join(ref_root, "Examples", ex, f + ".bin"), np.float32)

    np.savez_compressed(os.path.join(HERE, "mbir4d_reference.npz"), **out)
    print("wrote", os.path.join(HERE, "mbir4d_reference.npz"))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PHASECON_REFERENCE_ROOT", "")
    if not root:
        sys.exit("set PHASECON_REFERENCE_ROOT (or pass the path) to the phasecon checkout")
    main(root)
