"""The FP8 walk's query format, restated on the CPU: a query (times the rows'
per-dimension scales) is brought by a power of two so that its largest
magnitude lies in [128, 256), then stored as two E4M3 parts, hi = e4m3(x) and
lo = e4m3(x - hi) (prep_queries_kernel in pickle_b200/csrc/pk_fast.cu).  The
walk's one tensor-core product per k-step multiplies a row by both parts, so
the query's error is |hi + lo - x|.  This pins the precision the library's
comments and design notes state for it: 0.04% per component at the median and
0.2% at worst, against 2% for one E4M3 part - so the traversal's error is the
rows' E4M3 rounding, not the query's.  torch's float8_e4m3fn conversion rounds
to nearest even like the kernel's (saturation never applies below 256)."""
import numpy as np
import torch


def _split(x):
    m = np.abs(x).max(1, keepdims=True)
    pm = np.ldexp(1.0, 8 - np.frexp(m)[1]).astype(np.float32)  # largest |x| * pm in [128, 256)
    xs = x * pm
    t = torch.from_numpy(xs)
    hi = t.to(torch.float8_e4m3fn).float()
    lo = (t - hi).to(torch.float8_e4m3fn).float()
    return xs, hi.numpy(), lo.numpy()


def test_two_e4m3_parts_carry_the_query():
    rng = np.random.default_rng(0)
    for dim in (96, 128, 768):
        x = rng.standard_normal((1000, dim)).astype(np.float32)
        xs, hi, lo = _split(x)
        assert (np.abs(xs).max(1) >= 128).all() and (np.abs(xs).max(1) < 256).all()
        rel = np.abs(hi + lo - xs) / np.abs(xs)
        rel_hi = np.abs(hi - xs) / np.abs(xs)
        big = np.abs(xs) >= 1.0  # components above E4M3's subnormal range
        assert np.median(rel) < 5e-4, np.median(rel)
        assert rel[big].max() < 2.5e-3, rel[big].max()
        assert np.median(rel_hi) > 1e-2  # one part alone: about 2%
