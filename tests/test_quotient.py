"""The coarse solve's division by a divisor used many times (quotBy in
csrc/wig_device.cuh): a times the FP64 reciprocal of d, rounded to float,
must be IEEE's float quotient a / d bit for bit, NaNs compared as NaNs.

Checked on random bit patterns (every exponent: subnormals, zeros,
infinities and NaNs among them), on operands of one binade (quotients near
1, where rounding boundaries are closest), and on integer-valued operands,
against the host's IEEE division (numpy) and, on a B200, against the GPU's
float division (torch on CUDA)."""
import numpy as np
import pytest


def _cases(rng, n):
    bits = lambda: rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    yield bits(), bits()
    e = rng.integers(-60, 60, n)
    a = ((rng.random(n) + 1.0) * np.exp2(e)).astype(np.float32)
    d = ((rng.random(n) + 1.0) * np.exp2(e)).astype(np.float32)
    yield a, d
    yield rng.integers(-2 ** 24, 2 ** 24, n).astype(np.float32), rng.integers(1, 2 ** 12, n).astype(np.float32)
    sub = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1.1754942e-38, 3.4028235e38],
                   dtype=np.float32)
    yield np.repeat(sub, sub.size), np.tile(sub, sub.size)


def _same(q, r):
    qb, rb = q.view(np.uint32), r.view(np.uint32)
    return ((qb == rb) | (np.isnan(q) & np.isnan(r))).all()


def test_quotient_by_fp64_reciprocal_on_the_host():
    rng = np.random.default_rng(7)
    with np.errstate(all="ignore"):
        for a, d in _cases(rng, 1 << 21):
            q = (a / d).astype(np.float32)
            r = (a.astype(np.float64) * (1.0 / d.astype(np.float64))).astype(np.float32)
            assert _same(q, r)


@pytest.mark.gpu
def test_quotient_by_fp64_reciprocal_on_the_gpu():
    import torch
    rng = np.random.default_rng(11)
    for _ in range(8):
        for a, d in _cases(rng, 1 << 23):
            ta = torch.from_numpy(a).cuda()
            td = torch.from_numpy(d).cuda()
            q = (ta / td).cpu().numpy()
            r = (ta.double() * (1.0 / td.double())).float().cpu().numpy()
            assert _same(q, r)
