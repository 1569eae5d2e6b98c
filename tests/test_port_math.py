"""Accuracy of the bit-reproducible scalar math shared by the CPU restatement
and the kernels (oracle/port/orc_math.h; dr_device.cuh runs the same operation
sequences, which the GPU parity tests check bit for bit through the sky, phase
and free-flight code).  Against float64 references on dense samples of the
ranges the renderer feeds them: log on (0, 1] (free flights) and wider,
exp on the sky's arguments, sin/cos on [-2 pi, 2 pi] (sampling angles), x^1.5
and x^2.2 on the sky's and HG's bases.  The bound is 2 units in the last place
of the float32 result (for x^2.2 plus the conditioning of exp(2.2 log x))."""
import numpy as np
import pytest


def ulps(got, want):
    want32 = want.astype(np.float32)
    spacing = np.spacing(np.abs(want32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - want) / spacing


def test_log_exp_sincos_pow_within_two_ulps(port):
    rng = np.random.default_rng(4)
    u = ((np.arange(1 << 20, dtype=np.uint32) * 2 + 1) * 2.0 ** -21).astype(np.float32)  # the RNG's (2k+1) 2^-n
    x = np.concatenate([u, rng.uniform(1e-30, 1e6, 100000).astype(np.float32),
                        np.exp(rng.uniform(-80, 80, 100000)).astype(np.float32)])
    assert ulps(port.math_eval(0, x), np.log(x.astype(np.float64))).max() <= 2.0
    e = np.concatenate([rng.uniform(-80, 80, 200000), rng.uniform(-1, 1, 200000)]).astype(np.float32)
    assert ulps(port.math_eval(1, e), np.exp(e.astype(np.float64))).max() <= 2.0
    a = rng.uniform(-2 * np.pi, 2 * np.pi, 400000).astype(np.float32)
    a64 = a.astype(np.float64)
    # absolute error for sin/cos near their zeros, relative elsewhere
    for kind, f in ((2, np.sin), (3, np.cos)):
        got = port.math_eval(kind, a).astype(np.float64)
        assert (np.abs(got - f(a64)) <= 2.0 * np.spacing(np.maximum(np.abs(f(a64)), 2.0 ** -20).astype(np.float32))).all()
    b = np.concatenate([rng.uniform(0, 4, 200000), rng.uniform(0, 1e3, 100000)]).astype(np.float32)
    assert ulps(port.math_eval(4, b), b.astype(np.float64) ** 1.5).max() <= 2.0
    b = b[b > 1e-20]
    # x^2.2 = exp(2.2 log x): the rounding of the product 2.2 log x (half an ulp
    # of a number of size |2.2 ln x|) becomes that much relative error in the result
    allowed = 2.0 + 2.0 * np.abs(2.2 * np.log(b.astype(np.float64)))
    assert (ulps(port.math_eval(5, b), b.astype(np.float64) ** 2.2) <= allowed).all()
