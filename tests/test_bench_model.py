"""The benchmark's roofline byte model (CPU): the algorithmic bytes per
iteration kernel that bench.py divides by the measured times."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402

# 128^3 7-point stencil: n rows, z stored entries, the SELL layout's slots
# (every slice offset-uniform but 10 slots' worth), as the GPU plan reports them
N, Z = 2_097_152, 14_581_760
SLOTS, USLOTS = 14_614_528, 14_614_208


def test_index_bytes_of_the_offset_uniform_layout():
    ib = bench.index_bytes(N, 2, SLOTS, USLOTS)
    # 320 non-uniform slots at 2 bytes, one 4-byte offset per uniform entry
    # position, 12 bytes per slice
    assert ib == 2 * 320 + 4 * (USLOTS // 32) + 12 * (N // 32)
    assert 2.5e6 < ib < 2.7e6


def test_iteration_bytes_of_the_headline_form():
    ib = bench.index_bytes(N, 2, SLOTS, USLOTS)
    w_m, w_v, w_i = bench.form_widths(4)  # m_bf16: BF16 M, FP64 vectors
    assert (w_m, w_v, w_i) == (2, 8, 2)
    k = bench.bytes_per_kernel(N, Z, w_m, w_v, ib, True, w_a=4)
    names = bench.iteration_kernels(True)
    assert names == ["k_bi_p", "k_bi_y", "k_bi_ay", "k_bi_sz", "k_bi_az", "k_bi_xr"]
    by = dict(zip(names, k))
    # A's values at 4 bytes (its exact FP32 copy) in K2 and K4
    assert by["k_bi_ay"] == 4 * Z + ib + N * (8 + 2 * 8)
    assert by["k_bi_az"] == 4 * Z + ib + N * (16 + 8)
    # M's values at 2 bytes in K1b and K3
    assert by["k_bi_y"] == 2 * Z + ib + 2 * N * 8
    assert by["k_bi_sz"] == 2 * Z + ib + N * (24 + 8)
    # streaming kernels
    assert by["k_bi_p"] == N * (16 + 2 * 8)
    assert by["k_bi_xr"] == N * (40 + 3 * 8)
    # one iteration: 588 MB (705 MB with A's FP64 values)
    assert abs(sum(k) - 588.09e6) < 0.1e6
    k64 = bench.bytes_per_kernel(N, Z, w_m, w_v, ib, True)
    assert abs(sum(k64) - 704.74e6) < 0.1e6


def test_plain_form_iteration_bytes():
    ib = bench.index_bytes(N, 4, SLOTS, USLOTS)
    k = bench.bytes_per_kernel(N, Z, 8, 8, ib, False)
    assert bench.iteration_kernels(False)[0] == "k_bi_py"
    assert k[0] == 8 * Z + ib + N * (16 + 3 * 8)
    assert abs(sum(k) - 862.95e6) < 0.1e6
