"""Generate the golden fixtures in tests/golden/ from the reference SHTns 3.5.2
CPU library (built from the reference sources by oracle/Makefile into
oracle/_ref).

Run:  make -C oracle && python tests/golden/make_golden.py

Every case uses sht_quick_init, the reference's fixed (non-autotuned) kernel
choice, polar threshold 0, and inputs from tests/common.rand_spec with the
seed stored in the fixture, so the tests regenerate the inputs and compare
only outputs.  The spatial inputs of analysis-only cases are the reference's
own synthesis of the stored spectral recipe.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import shtns_ref as R  # noqa: E402
from common import rand_spec  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")

# name: (lmax, mmax, mres, nlat, nphi, norm, layout, ltr, kind)
CASES = {
    "cfg1_scalar": (127, 127, 1, 192, 384, R.sht_orthonormal, R.SHT_THETA_CONTIGUOUS, None, "scalar"),
    "small_sphtor": (31, 31, 1, 48, 64, R.sht_orthonormal, R.SHT_THETA_CONTIGUOUS, None, "sphtor"),
    "small_qst": (31, 31, 1, 48, 64, R.sht_orthonormal, R.SHT_THETA_CONTIGUOUS, None, "qst"),
    "phi_schmidt_mres2": (40, 16, 2, 64, 96, R.sht_schmidt, R.SHT_PHI_CONTIGUOUS, None, "qst"),
    "fourpi_nocs_ltr": (47, 40, 1, 72, 96, R.sht_fourpi | R.SHT_NO_CS_PHASE, R.SHT_THETA_CONTIGUOUS, 30, "qst"),
    "realnorm_south": (33, 33, 1, 50, 72, R.sht_orthonormal | R.SHT_REAL_NORM,
                       R.SHT_THETA_CONTIGUOUS | R.SHT_SOUTH_POLE_FIRST, None, "qst"),
}


def make_case(name, case, seed):
    lmax, mmax, mres, nlat, nphi, norm, layout, ltr, kind = case
    ref = R.RefSHT(lmax, mmax, mres, norm, nlat, nphi, flags=R.sht_quick_init | layout, eps=0.0, nthreads=1)
    out = {}
    q = rand_spec(lmax, mmax, mres, seed, power=1.0)
    s = rand_spec(lmax, mmax, mres, seed + 1, power=1.5, zero_l0=True)
    t = rand_spec(lmax, mmax, mres, seed + 2, power=1.5, zero_l0=True)
    if kind == "scalar":
        v = ref.synth(q, ltr)
        out["synth_v"] = v
        out["analys_q"] = ref.analys(v, ltr)
    elif kind == "sphtor":
        vt, vp = ref.sphtor_synth(s, t, ltr)
        out["synth_vt"], out["synth_vp"] = vt, vp
        out["analys_s"], out["analys_t"] = ref.sphtor_analys(vt, vp, ltr)
    else:
        vr, vt, vp = ref.qst_synth(q, s, t, ltr)
        out["synth_vr"], out["synth_vt"], out["synth_vp"] = vr, vt, vp
        out["analys_q"], out["analys_s"], out["analys_t"] = ref.qst_analys(vr, vt, vp, ltr)
    out["ct"] = ref.ct
    ref.close()
    meta = dict(lmax=lmax, mmax=mmax, mres=mres, nlat=nlat, nphi=nphi, norm=norm, layout=layout,
                ltr=ltr, kind=kind, seed=seed)
    return meta, out


def main():
    index = {}
    for i, (name, case) in enumerate(CASES.items()):
        seed = 1000 + 10 * i
        meta, arrays = make_case(name, case, seed)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrays)
        index[name] = meta
        print(name, {k: v.shape for k, v in arrays.items()})
    with open(os.path.join(OUT, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
