"""GPU: CUDA-graph replay of the level schedule (full factorization) and of the
solve sweeps / preconditioner applications is used and changes nothing: the
results are bit-identical to direct launches (MFGPU_GRAPHS=0)."""
import numpy as np
import pytest

from mfgpu import MF2D, MF3D, MFBatch, MFGPU_MIXED, stencil
from problems import problem

pytestmark = pytest.mark.gpu


def _run(make, b, monkeypatch, graphs):
    monkeypatch.setenv("MFGPU_GRAPHS", "1" if graphs else "0")
    F = make()
    out = []
    for _ in range(3):           # captured on the second run, replayed on the third
        F.Factor()
        out.append(F.Solve(b))
        out.append(F.Solve(b))
    g = F.graphs()
    F.close()
    return out, g


@pytest.mark.parametrize("case", ["2d-fp64", "3d-mixed", "2d-coop-sweeps"])
def test_graph_replay_is_bit_identical(case, monkeypatch):
    if case == "3d-mixed":
        N = (31, 31, 31)
        _, A, b = problem(3, N, seed=51, nrhs=2)
        make = lambda: MF3D(A, N[0], N[1], N[2], 1, 4, precision=MFGPU_MIXED)
    else:
        N = (255, 255)
        _, A, b = problem(2, N, seed=52, nrhs=3)
        if case == "2d-coop-sweeps":
            monkeypatch.setenv("MFGPU_SOLVE_COOP_MIN_N", "256")
        make = lambda: MF2D(A, N[0], N[1], 1, 4)
    on, g_on = _run(make, b.T, monkeypatch, True)
    off, g_off = _run(make, b.T, monkeypatch, False)
    assert g_on[0] and g_on[1] >= 1, g_on          # both kinds of graph were captured
    assert g_off == (False, 0)
    for x, y in zip(on, off):
        np.testing.assert_array_equal(x, y)


def test_batch_graph_replay(monkeypatch):
    probs, rhs = [], []
    for i, side in enumerate((63, 127, 63)):
        N = (side, side)
        _, A, b = problem(2, N, seed=60 + i, nrhs=2)
        probs.append((A, N, 1, 4))
        rhs.append(b.T)
    res = {}
    for graphs in (True, False):
        monkeypatch.setenv("MFGPU_GRAPHS", "1" if graphs else "0")
        F = MFBatch(probs)
        B = F.join(rhs, 2)
        xs = []
        for _ in range(3):
            F.Factor()
            xs.append(F.Solve(B))
        res[graphs] = (xs, F.graphs())
        F.close()
    assert res[True][1][0] and not res[False][1][0]
    for x, y in zip(res[True][0], res[False][0]):
        np.testing.assert_array_equal(x, y)
