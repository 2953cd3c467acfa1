"""Committed golden vectors from the compiled reference (tests/golden/
make_golden.py) against the oracle restatement (CPU) and the sm_100a
library (GPU).  These run without the compiled reference present."""
import json
import os

import numpy as np
import pytest

from oracle.pyoracle import OracleModel
from profit_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cases.npz")


def _cases():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


def _build(M, entry):
    if "profile" in entry:
        m = M(entry["width"], entry["height"])
        m.add_profile(entry["profile"], **entry["params"])
        return m
    if entry["workload"] == "single_sersic":
        wl = W.single_sersic(seed_tag=entry["seed_tag"])
    else:
        wl = W.bulge_disk_ps(width=entry["width"], height=entry["height"], psf_size=entry["psf_size"])
    return W.configure(M(wl["width"], wl["height"]), wl)


def test_restatement_matches_golden():
    z, meta = _cases()
    for entry in meta:
        m = _build(OracleModel, entry)
        img, _ = m.evaluate()
        ref = z[entry["key"] + "_image"]
        if "profile" in entry:
            assert np.array_equal(img, ref), entry["key"]
            assert m.level_counts(0) == list(z[entry["key"] + "_levels"]), entry["key"]
        else:
            assert np.max(np.abs(img - ref)) <= 1e-13 * np.max(np.abs(ref)), entry["key"]


@pytest.mark.gpu
def test_library_fp64_matches_golden():
    from profit_b200 import Model
    z, meta = _cases()
    for entry in meta:
        m = _build(Model, entry)
        m.set_debug(True)
        img, _ = m.evaluate()
        ref = z[entry["key"] + "_image"]
        assert np.max(np.abs(img - ref)) <= 1e-12 * np.max(np.abs(ref)), entry["key"]
        if "profile" in entry:
            assert m.level_counts(0) == list(z[entry["key"] + "_levels"]), entry["key"]
