"""Generates the golden fixtures in tests/golden from the reference's OWN CPU
kernels (oracle/_ref/libbgprtm_ref.so, compiled from the reference tree by
oracle/Makefile).  Run here, where the reference tree exists:

    python tests/golden/make_golden.py

Inputs are regenerated in the tests from the seeds stored in each fixture
(numpy's default_rng is platform independent); only the reference outputs
are stored.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from tests.golden_inputs import CASES, ILLUM_SMOOTH, case_inputs, codec_input, illum_input, spread_cases  # noqa: E402


def main():
    if not O.ref_available():
        O.build()
    out = {}
    for name, c in CASES.items():
        spec, model, w0, w1 = case_inputs(c)
        r = O.Reference(spec, nthreads=1)
        r.set_model(**model)
        r.put(0, w0)
        r.put(1, w1)
        for _ in range(c["steps"]):
            r.kernel()
            r.update2nd()
            r.swap()
        out[f"{name}__w1"] = r.get(1).reshape(spec.shape)
        r.close()
    # COMPRESS_16 codec: wavefield-like and edge-case inputs, codes and decode
    for cname, (a, nx, ny, nz) in codec_input().items():
        codes = O.ref_c16_compress(a, nx, ny, nz)
        out[f"c16_{cname}__codes"] = codes
        out[f"c16_{cname}__decoded"] = O.ref_c16_uncompress(codes, nx, ny, nz)
    # compact FD plans and the PML profile
    for n in (40, 57):
        for s in (0, 1):
            bm, bl, am = O.ref_cfd_plan(n, 10.0, s)
            out[f"cfd_plan_{n}_{s}__bm"], out[f"cfd_plan_{n}_{s}__bl"], out[f"cfd_plan_{n}_{s}__am"] = bm, bl, am
    # spread kernels: Util::CompactOrmsbySpreadCoeff
    offs, coefs = [], []
    for n, x, k1, k2, nl, dip in spread_cases():
        o, c = O.ref_spread_coeffs(n, x, k1, k2, nl, dip)
        offs.append((o, len(c)))
        coefs.append(np.pad(c, (0, 40 - len(c))))
    out["spread_offsets"] = np.array(offs, np.int32)
    out["spread_coeffs"] = np.array(coefs, np.float32)
    # illumination smoothing: volumefilter.cpp's running box averages
    for name, (shape, hxy, hz) in ILLUM_SMOOTH.items():
        out[f"illum_smooth_{name}"] = O.ref_avg_volume(illum_input(name), hxy, hz)
    out["pml_coef_20"] = O.ref_pml_coef(128, 20, 10.0, 0.001, 4500.0)
    out["pml_coef_32"] = O.ref_pml_coef(512, 32, 10.0, 0.0007, 4500.0)
    np.savez_compressed(os.path.join(HERE, "reference_kernels.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
