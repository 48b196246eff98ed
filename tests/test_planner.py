"""The engine's planner, executed on the CPU by the test interpreter.

tests/native/plan_emulator.cpp links the product planner (plan.cpp) and runs
each planned launch on the host with the generated addition code, in a
NaN-poisoned workspace.  Its result must equal the CPU oracle bit for bit
for every algorithm, shape, alpha/beta and DFS/BFS/HYBRID split.
"""

import ctypes

import numpy as np
import pytest

import oracle
from helpers import emulator

P = ctypes.POINTER(ctypes.c_double)
L_ORACLE = oracle.oracle_lib()
NAMES = [L_ORACLE.oracle_algorithm_name(i).decode() for i in range(L_ORACLE.oracle_num_algorithms())]
APPROX = {"bini322_10_52_approx", "schonhage333_21_117_approx", "smirnov333_20_182_approx"}

SHAPES = [
    (57, 40, 35, 2, 1.0, 0.0),
    (64, 64, 64, 2, 1.0, 0.0),
    (101, 80, 74, 1, 7.0, -1.3),
    (30, 33, 29, 3, -1.2, 2.5),
    (7, 5, 3, 2, 1.0, 0.5),    # blocks of size zero: everything by peeling
    (19, 23, 17, 0, 2.0, 3.0),  # num_steps 0: one product, beta ignored
]


def run_emu(E, idx, A, B, C, steps, x, alpha, beta, d):
    m, k = A.shape
    n = B.shape[1]
    stats = (ctypes.c_int64 * 5)()
    rc = E.emu_fast_matmul(idx, A.ctypes.data_as(P), m, B.ctypes.data_as(P), k, C.ctypes.data_as(P), m, m, k, n,
                           steps, x, alpha, beta, d, stats)
    assert rc == 0
    return list(stats)


@pytest.mark.parametrize("alg", NAMES)
def test_planner_matches_oracle_bit_exact(alg):
    E = emulator()
    idx = NAMES.index(alg)
    for si, (m, k, n, steps, alpha, beta) in enumerate(SHAPES):
        A = oracle.uniform(m, k, si, 1)
        B = oracle.uniform(k, n, si, 2)
        C0 = oracle.uniform(m, n, si, 3)
        x = 1e-4 if alg in APPROX else 1e-8
        want = C0.copy(order="F")
        oracle.fast_matmul(alg, A, B, want, steps, x, alpha, beta)
        for d in range(steps + 1):
            got = C0.copy(order="F")
            run_emu(E, idx, A, B, got, steps, x, alpha, beta, d)
            assert not np.isnan(got).any() or np.isnan(want).any()
            assert np.array_equal(want, got, equal_nan=True), (alg, m, k, n, steps, d)


def test_breadth_first_groups_each_level_into_one_launch():
    E = emulator()
    idx = NAMES.index("strassen")
    A = oracle.uniform(64, 64, 1, 1)
    B = oracle.uniform(64, 64, 1, 2)
    C = np.zeros((64, 64), order="F")
    s_bfs = run_emu(E, idx, A, B, C, 2, 1e-8, 1.0, 0.0, 0)
    s_dfs = run_emu(E, idx, A, B, C, 2, 1e-8, 1.0, 0.0, 2)
    # BFS: one formation + one combination per level, one leaf GEMM launch
    assert s_bfs[:3] == [2, 1, 2] and s_bfs[3] == 49
    # DFS: 1 + 7 formations, 7 leaf launches (7 leaves each), 7 + 1 combinations
    assert s_dfs[:3] == [8, 7, 8] and s_dfs[3] == 49
    assert s_bfs[4] > s_dfs[4]


def test_workspace_scales_with_breadth_first_levels():
    E = emulator()
    idx = NAMES.index("grey424_26_206")
    sizes = [E.emu_workspace_bytes(idx, 16384, 16384, 16384, 3, d) for d in range(4)]
    # the root level has one sub-problem, so one depth-first level plans like BFS
    assert sizes[0] == sizes[1] > sizes[2] > sizes[3] > 0
    # the reference's MemoryManager needs ~209.7 GiB here; pure DFS needs a small fraction
    assert sizes[3] < 20 * 2**30


def test_batch_program_matches_oracle_per_item():
    """Mixed batch (algorithms, depths, odd shapes): every item equals its own
    oracle call bit for bit, and all leaves share one GEMM launch."""
    E = emulator()
    rng = np.random.default_rng(3)
    names = ["strassen", "grey424_26_206", "grey333_23_125", "classical222_8_24", "smirnov333_23_128"]
    specs = []
    for i in range(14):
        alg = names[i % len(names)]
        steps = [0, 1, 2][i % 3]
        m, k, n = (int(v) for v in rng.integers(5, 70, size=3))
        specs.append((alg, steps, m, k, n))
    a_off, b_off, c_off, dims, algs, steps = [], [], [], [], [], []
    ta = tb = tc = 0
    for alg, s, m, k, n in specs:
        a_off.append(ta); b_off.append(tb); c_off.append(tc)
        ta += m * k; tb += k * n; tc += m * n
        dims += [m, k, n]; algs.append(NAMES.index(alg)); steps.append(s)
    A = oracle.uniform(ta, 1, 8, 1).ravel()
    B = oracle.uniform(tb, 1, 8, 2).ravel()
    C0 = oracle.uniform(tc, 1, 8, 3).ravel()
    C = C0.copy()
    i64 = ctypes.c_int64
    arr = lambda t, v: (t * len(v))(*v)
    stats = (i64 * 5)()
    rc = E.emu_fast_matmul_batch(len(specs), arr(ctypes.c_int, algs), arr(ctypes.c_int, steps), arr(i64, dims),
                                 A.ctypes.data_as(P), arr(i64, a_off), B.ctypes.data_as(P), arr(i64, b_off),
                                 C.ctypes.data_as(P), arr(i64, c_off), 1e-8, 1.25, 0.5, stats)
    assert rc == 0
    assert stats[1] == 1  # one leaf GEMM launch for the whole batch
    for i, (alg, s, m, k, n) in enumerate(specs):
        Ai = np.asfortranarray(A[a_off[i]:a_off[i] + m * k].reshape(k, m).T)
        Bi = np.asfortranarray(B[b_off[i]:b_off[i] + k * n].reshape(n, k).T)
        want = np.asfortranarray(C0[c_off[i]:c_off[i] + m * n].reshape(n, m).T)
        oracle.fast_matmul(alg, Ai, Bi, want, s, 1e-8, 1.25, 0.5)
        got = np.asfortranarray(C[c_off[i]:c_off[i] + m * n].reshape(n, m).T)
        assert np.array_equal(want, got), (i, alg, s, m, k, n)


def test_even_blocks_agree_across_schedules_and_with_the_oracle():
    """Block rows and inner dimensions of 256 or more are made even (one more
    row or inner index peeled), so 1031 x 1030 x 1029 splits as 1031 -> 514
    -> 256 where the reference's floor splitting gives 515 -> 257: the
    programs differ from the oracle's recursion, every depth-first split of
    them gives the same bits, and the result stays within rounding of the
    oracle's."""
    E = emulator()
    idx = NAMES.index("strassen")
    m, k, n = 1031, 1030, 1029
    A = oracle.uniform(m, k, 41, 1)
    B = oracle.uniform(k, n, 41, 2)
    C0 = oracle.uniform(m, n, 41, 3)
    want = C0.copy(order="F")
    oracle.fast_matmul("strassen", A, B, want, 2, 1e-8, 1.25, -0.5)
    got = []
    for d in range(3):
        C = C0.copy(order="F")
        run_emu(E, idx, A, B, C, 2, 1e-8, 1.25, -0.5, d)
        got.append(C)
    for C in got[1:]:
        assert np.array_equal(C, got[0])
    assert float(np.abs(got[0] - want).max() / np.abs(want).max()) <= 1e-13
