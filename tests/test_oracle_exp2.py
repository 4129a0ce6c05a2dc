"""The blend's deterministic 2^y: accuracy of the oracle's restatement, its
special cases, and that the coefficients in the oracle and in the CUDA
header are the ones oracle/fit_exp2.py derives (CPU only; the GPU tests
check the kernels against the oracle bit for bit through the images)."""
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exp2_det_relative_error(orc):
    rng = np.random.default_rng(5)
    y = np.concatenate([rng.uniform(-124.9, 122.9, 200000), rng.uniform(-0.5, 0.5, 200000),
                        np.arange(-124, 123) + rng.uniform(-0.5, 0.5, 247)]).astype(np.float32)
    got = orc.exp2_det(y).astype(np.float64)
    want = np.exp2(y.astype(np.float64))
    assert np.max(np.abs(got / want - 1.0)) < 2.3e-7


def test_exp2_det_special_values(orc):
    n = np.arange(-124, 123, dtype=np.float32)
    assert np.array_equal(orc.exp2_det(n), np.exp2(n.astype(np.float64)).astype(np.float32))  # exact powers
    out = orc.exp2_det(np.array([-125.0, -1e30, 123.0, 1e30, np.nan, -np.inf, np.inf], np.float32))
    assert out[0] == 0 and out[1] == 0 and np.isinf(out[2]) and np.isinf(out[3]) and np.isnan(out[4])
    assert out[5] == 0 and np.isinf(out[6])


def test_exp2_coefficients_come_from_the_fit():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import fit_exp2
    finally:
        sys.path.pop(0)
    c, err = fit_exp2.fit()
    assert err < 7e-8
    want = [float(np.float32(v)) for v in c]  # c1..c5
    src = open(os.path.join(ROOT, "oracle", "oracle.cpp")).read()
    body = src[src.index("inline float exp2_det_f32"):]
    body = body[:body.index("\n}\n")]
    cpu = [float(x) for x in re.findall(r"([0-9.]+e?-?[0-9]*)f\)?;", body) if float(x) < 1.0 and "." in x]
    assert [float(np.float32(v)) for v in cpu[:5]] == want[::-1]
    hdr = open(os.path.join(ROOT, "del-splat_b200", "csrc", "common.cuh")).read()
    gpu = {int(k): float(v) for k, v in re.findall(r"kExp2C(\d) = ([0-9.e-]+)f", hdr)}
    assert [float(np.float32(gpu[j])) for j in range(1, 6)] == want
