"""The operand splits of the tensor-core GEMMs, restated in numpy (no GPU).

The packers split FP32 values into planes of 16-bit floats, each plane the round-to-nearest value of the
remainder left by the previous ones, and the GEMMs sum the plane products. In FP32 arithmetic each
remainder is exact, so three bf16 planes hold an FP32 value exactly as long as the remainders stay
normal (|x| >= 2^-100, far below any operand of the path; smaller values are off by at most the bf16
subnormal spacing 2^-133), and two fp16 planes hold values of magnitude up to 2^14 to about 2^-22
relative (the pass scales its FP16x2 operand into that range).
"""
import numpy as np


def bf16_rne(x):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def split(x, rnd, nplanes):
    planes, r = [], np.asarray(x, dtype=np.float32)
    for _ in range(nplanes):
        p = rnd(r)
        planes.append(p)
        r = (r - p).astype(np.float32)  # exact in FP32
    return planes


def test_bf16x3_split_is_exact_for_fp32():
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.standard_normal(200000), rng.standard_normal(20000) * 1e-30,
                        rng.standard_normal(20000) * 1e30, [0.0, 1.0, -1.0, 3.0e-38]]).astype(np.float32)
    planes = split(x, bf16_rne, 3)
    # the planes add up to the FP32 value exactly (summed in FP64 to see every bit)
    total = sum(p.astype(np.float64) for p in planes)
    normal = np.abs(x) >= 2.0 ** -100
    np.testing.assert_array_equal(total[normal], x[normal].astype(np.float64))
    assert np.abs(total[~normal] - x[~normal].astype(np.float64)).max() <= 2.0 ** -133


def test_fp16x2_split_accuracy_in_range():
    rng = np.random.default_rng(6)
    x = (rng.uniform(-1, 1, 200000) * 2.0 ** 14).astype(np.float32)
    planes = split(x, lambda r: r.astype(np.float16).astype(np.float32), 2)
    total = sum(p.astype(np.float64) for p in planes)
    rel = np.abs(total - x.astype(np.float64)) / np.maximum(np.abs(x.astype(np.float64)), 1e-30)
    big = np.abs(x) > 1.0  # away from fp16's subnormal range for the remainder plane
    assert rel[big].max() <= 2.0 ** -21
