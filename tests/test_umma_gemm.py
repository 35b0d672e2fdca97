"""The learned initialiser's GEMM kernels: the sm_100a tensor-core kernel (TMA
tile loads, tcgen05.mma into tensor memory, tcgen05.ld epilogue) and the
warp-level mma.sync kernel it replaces.

Both multiply BF16 operands with FP32 accumulation, so each is checked against
the FP64 product of the same BF16 values (oracle/mlp_oracle.py's rounding) with
a bound of FP32 summation error, and against each other.  The shapes are the
ones training and inference use (batch x 256 x 256, the 32-wide output layer,
the split-K weight gradients with a reduction over the batch) plus ragged ones:
rows that are not a multiple of the 128-row tile, reductions shorter than the
64-value stage (read as zeros past the end), more than 256 columns.  Small
grids take narrower column tiles (down to 32), so both tile widths appear.
"""
import numpy as np
import pytest

import me_b200
from oracle import mlp_oracle as mo


def bf16_bits(x):
    """BF16 bit patterns (uint16) of FP32 values, rounded to nearest even."""
    return (mo.bf16_round(x).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def bf16_values(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def operands(m, n, r, seed):
    rng = np.random.default_rng(seed)
    a = bf16_bits(rng.normal(0, 1, (m, r)).astype(np.float32))
    bt = bf16_bits(rng.normal(0, 1 / np.sqrt(r), (n, r)).astype(np.float32))
    return a, bt


def check_product(y, a, bt, bias=None, gelu=False, z=None):
    """y (and z) against the FP64 product of the BF16 operands; the bound is
    FP32 rounding of a length-r sum of terms of magnitude |a| |b|."""
    A, B = bf16_values(a), bf16_values(bt)
    ref = A @ B.T
    scale = np.abs(A) @ np.abs(B).T
    if bias is not None:
        ref = ref + bias[None, :].astype(np.float64)
        scale = scale + np.abs(bias)[None, :]
    tol = 4e-6 * scale + 1e-30
    if z is not None:
        assert np.all(np.abs(z - ref) <= tol), np.max(np.abs(z - ref) / tol)
    want = mo.gelu(ref) if gelu else ref
    assert np.all(np.abs(y - want) <= tol + 2e-6 * np.abs(want)), np.max(np.abs(y - want) / tol)


# ---------------------------------------------------------------- CPU ------

def test_gemm_argument_checks():
    L = me_b200.lib()
    a, bt = operands(4, 4, 32, 0)
    y = np.zeros((4, 4), dtype=np.float32)
    u16 = me_b200.ctypes.POINTER(me_b200.ctypes.c_uint16)
    f32 = me_b200.ctypes.POINTER(me_b200.ctypes.c_float)
    pa, pb = a.ctypes.data_as(u16), bt.ctypes.data_as(u16)
    py = y.ctypes.data_as(f32)
    for path, m, n, r, split in [(2, 4, 4, 32, 1), (0, 4, 4, 24, 1), (0, 0, 4, 32, 1),
                                 (0, 4, 4, 32, 2), (0, 4, 4, 64, 0)]:
        assert L.me_gemm_bf16(0, path, pa, pb, m, n, r, split, None, 0, None, py,
                              None) == me_b200.ME_ERR_ARG
    assert L.me_gemm_bf16(0, 0, None, pb, 4, 4, 32, 1, None, 0, None, py,
                          None) == me_b200.ME_ERR_ARG
    assert L.me_mlp_set_gemm(None, 0) == me_b200.ME_ERR_ARG


# ---------------------------------------------------------------- GPU ------

SHAPES = [  # m, n, r, split
    (4096, 256, 256, 1),    # hidden layer of a training batch
    (65536, 256, 256, 1),   # hidden layer of an inference chunk
    (4096, 32, 256, 1),     # output layer
    (4096, 256, 32, 1),     # first layer of a 6-wavelength grid: r < 64
    (300, 256, 96, 1),      # ragged rows, r not a multiple of 64
    (200, 272, 128, 1),     # small grid: 32-wide column tiles, the last 16 wide
    (40000, 272, 64, 1),    # 256-wide column tiles, the second 16 wide
    (77, 48, 224, 1),       # fewer rows than one tile
    (256, 256, 4096, 16),   # weight gradient: reduction over the batch, split 16
    (32, 256, 4096, 16),    # output-layer weight gradient (32 rows)
    (256, 256, 4096, 4),
]


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,r,split", SHAPES)
def test_tcgen05_gemm_vs_fp64(m, n, r, split):
    a, bt = operands(m, n, r, m + n + r)
    z, y, ran = me_b200.gemm_bf16(a, bt, "tcgen05", split=split)
    assert ran == "tcgen05"
    check_product(y, a, bt)
    if z is not None:
        check_product(z, a, bt)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,r", [(4096, 256, 256), (300, 256, 96), (4096, 32, 256)])
def test_tcgen05_epilogue_bias_gelu(m, n, r):
    a, bt = operands(m, n, r, 7)
    bias = np.random.default_rng(8).normal(0, 0.5, n).astype(np.float32)
    z, y, ran = me_b200.gemm_bf16(a, bt, "tcgen05", bias=bias, gelu=True)
    assert ran == "tcgen05"
    check_product(y, a, bt, bias=bias, gelu=True, z=z)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,r,split", [(4096, 256, 256, 1), (200, 272, 128, 1),
                                         (256, 256, 4096, 16)])
def test_tcgen05_agrees_with_mma_sync(m, n, r, split):
    a, bt = operands(m, n, r, 3)
    _, y0, ran0 = me_b200.gemm_bf16(a, bt, "tcgen05", split=split)
    _, y1, ran1 = me_b200.gemm_bf16(a, bt, "mma_sync", split=split)
    assert (ran0, ran1) == ("tcgen05", "mma_sync")
    check_product(y1, a, bt)
    A, B = bf16_values(a), bf16_values(bt)
    bound = 8e-6 * (np.abs(A) @ np.abs(B).T)
    assert np.all(np.abs(y0 - y1) <= bound)


@pytest.mark.gpu
def test_shapes_outside_the_tensor_core_kernel_run_on_mma_sync():
    a, bt = operands(256, 40, 64, 5)  # 40 columns: not a multiple of 16
    _, y, ran = me_b200.gemm_bf16(a, bt, "tcgen05")
    assert ran == "mma_sync"
    check_product(y, a, bt)
    a, bt = operands(256, 256, 1024, 6)  # split 32: shares of 32, not 64
    _, y, ran = me_b200.gemm_bf16(a, bt, "tcgen05", split=32)
    assert ran == "mma_sync"
    check_product(y, a, bt)
