"""The tcgen05.mma kind::tf32 instruction rate on this device (tci_selftest_mma_rate): cycles per
instruction for M = 64 / 128, N = 64 / 128 / 256 and 1, 2 or 4 independent accumulators, issued back to back
by one thread per SM.  Prints the table; checks that every run completed and that interleaving
independent accumulators does not slow the issue down."""
import ctypes as C

import pytest

from tigerci_b200._lib import lib

pytestmark = pytest.mark.gpu


def test_mma_instruction_rate_table(need_gpu):
    L = lib()
    rows = []
    for m in (128, 64):
        for n in (64, 128, 256):
            for nacc in (1, 2, 4):
                if n * nacc * (2 if m == 64 else 1) > 512:
                    continue
                cyc = C.c_double(0.0)
                assert L.tci_selftest_mma_rate(0, m, n, nacc, 512, C.byref(cyc)) == 0
                flops = 2.0 * m * n * 8
                rows.append((m, n, nacc, cyc.value, flops / cyc.value))
    print("\nM, N, accumulators, cycles per MMA, TF32 flops per cycle per SM")
    for m, n, nacc, cyc, fpc in rows:
        print(f"{m}, {n}, {nacc}, {cyc:.1f}, {fpc:.0f}")
    by = {(m, n, a): c for m, n, a, c, _ in rows}
    for (m, n, a), c in by.items():
        if a == 2:
            assert c <= by[(m, n, 1)] * 1.05
