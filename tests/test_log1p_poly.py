"""CPU check of the FMA polynomial the tensor-core logistic pass uses for
log(1 + e), e in [0, 1] (the softplus of the log-likelihood,
bayes_logreg.jl:118-154): the coefficients are read from the kernel source and
evaluated with FP32 fused multiply-adds, emulated exactly in FP64."""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "parallelmcmc.jl_b200", "csrc",
                   "logistic_tc.cu")


def _coefficients():
    s = open(SRC).read()
    body = s[s.index("float log1p_unit(float e)"):]
    body = body[:body.index("return e * q;")]
    nums = re.findall(r"(-?\d+\.\d+(?:e-?\d+)?)f", body)
    return [np.float32(float(x)) for x in nums]  # highest degree first


def _fma32(a, b, c):
    # a * b is exact in FP64 for FP32 inputs; one rounding of the sum to FP64
    # and one to FP32 (the double rounding is immaterial at this bound)
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def test_log1p_poly_error_bound():
    c = _coefficients()
    assert len(c) == 10 and c[-1] == np.float32(1.0)
    e = np.linspace(0.0, 1.0, 400001).astype(np.float32)
    q = np.full_like(e, c[0])
    for k in c[1:]:
        q = _fma32(q, e, np.full_like(e, k))
    v = (e * q).astype(np.float32)
    err = np.abs(v.astype(np.float64) - np.log1p(e.astype(np.float64)))
    assert err.max() < 1.3e-7
    # relative accuracy near 0, where log1p(e) ~ e
    small = e[1:2001]
    rel = err[1:2001] / np.log1p(small.astype(np.float64))
    assert rel.max() < 1e-6
