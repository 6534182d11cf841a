"""The emission kernel (lumen_b200/csrc/project.cu, emit_kernel) splits an
instance's offset q inside its splat's tile rectangle into a row and a column
with a float reciprocal of the rectangle width w and one integer correction
step, for q < 2^20 (plain integer division beyond). This checks, in IEEE
float32 arithmetic identical to the kernel's (round-to-nearest reciprocal and
product, truncating conversion), that the row always equals q // w: around
every multiple of w and on random pairs."""
import numpy as np

LIMIT = 1 << 20


def kernel_row(q, w):
    q = q.astype(np.uint64)
    w = w.astype(np.uint64)
    rcp = np.float32(1.0) / w.astype(np.float32)
    row = np.trunc(q.astype(np.float32) * rcp).astype(np.uint64)
    dec = row * w > q
    row = np.where(dec, row - 1, row)
    inc = (~dec) & ((row + 1) * w <= q)
    return np.where(inc, row + 1, row)


def test_row_exact_around_multiples():
    for w in list(range(1, 600)) + [1023, 1024, 1025, 4095, 4096, 8191, 65535]:
        k = np.arange(0, LIMIT // w + 2, dtype=np.uint64)
        q = np.concatenate([k * w, k * w + w - 1, k * w + 1])
        q = q[q < LIMIT]
        w_arr = np.full(q.shape, w, np.uint64)
        np.testing.assert_array_equal(kernel_row(q, w_arr), q // w_arr)


def test_row_exact_random():
    rng = np.random.default_rng(7)
    q = rng.integers(0, LIMIT, 4_000_000, dtype=np.uint64)
    for hi in (64, 1 << 12, 1 << 16):
        w = rng.integers(1, hi, q.shape[0], dtype=np.uint64)
        np.testing.assert_array_equal(kernel_row(q, w), q // w)
