"""Writes tests/golden/reference_cases.npz: model images of small cases
computed by the reference's own libprofit C++ (compiled in place by
oracle/Makefile, oracle/_ref/libprofit_ref.so) plus per-level subsampling
counts from its PROFIT_DEBUG build.  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

The fixtures let parity be checked where the compiled reference is absent.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.pyoracle import RefModel  # noqa: E402
from profit_b200 import workloads as W  # noqa: E402
from test_oracle import PROFILE_CASES  # noqa: E402


def main():
    out = {}
    meta = []
    for i, (name, params) in enumerate(PROFILE_CASES):
        m = RefModel(100, 100)
        m.add_profile(name, **params)
        img, _ = m.evaluate()
        d = RefModel(100, 100, debug=True)
        d.set_omp_threads(1)
        d.add_profile(name, **params)
        d.evaluate()
        out[f"case{i}_image"] = img
        out[f"case{i}_levels"] = np.array(d.integrations(0), dtype=np.int64)
        meta.append({"key": f"case{i}", "profile": name, "params": params, "width": 100, "height": 100})
    wl = W.single_sersic()
    m = W.configure(RefModel(wl["width"], wl["height"]), wl)
    img, _ = m.evaluate()
    out["single_sersic_image"] = img
    meta.append({"key": "single_sersic", "workload": "single_sersic", "seed_tag": 1})
    wl = W.bulge_disk_ps(width=160, height=140, psf_size=25)
    m = W.configure(RefModel(wl["width"], wl["height"]), wl)
    img, _ = m.evaluate()
    out["bulge_disk_ps_small_image"] = img
    meta.append({"key": "bulge_disk_ps_small", "workload": "bulge_disk_ps", "width": 160, "height": 140,
                 "psf_size": 25})
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz"), **out)


if __name__ == "__main__":
    main()
