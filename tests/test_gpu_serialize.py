"""GPU: factor serialisation (mfgpu_save / mfgpu_load).

A factorization written by save() and read by load() into a fresh handle of
the same problem must behave exactly like the original: its solves, applies
and a localized update afterwards are bit-identical to the original handle's.
Files of another problem, of the other precision, or with a corrupted payload
are rejected with MFGPU_ERR_ARG (ValueError in Python, as every argument
error), and saving before Factor() with MFGPU_ERR_STATE.
"""
import numpy as np
import pytest

from mfgpu import MF2D, MF3D, MFGPU_MIXED, MFError, _lib, stencil
from problems import patch_update, problem

pytestmark = pytest.mark.gpu


def make(N, A, **kw):
    return MF2D(A, N[0], N[1], 1, 4, **kw) if len(N) == 2 else MF3D(A, N[0], N[1], N[2], 1, 4, **kw)


@pytest.mark.parametrize("N,precision", [((63, 63), None), ((15, 15, 15), None),
                                         ((63, 63), MFGPU_MIXED), ((31, 31, 31), MFGPU_MIXED)])
def test_loaded_factor_equals_original(N, precision, tmp_path):
    kw = {} if precision is None else {"precision": precision}
    a, A, b = problem(len(N), N, seed=61, nrhs=2)
    F = make(N, A, **kw)
    F.Factor()
    path = tmp_path / "factor.mfgpu"
    F.save(path)
    G = make(N, A, **kw)                      # built for the same problem, never factored
    G.load(path)
    assert np.array_equal(G.Solve(b.T), F.Solve(b.T))
    x = b[0]
    assert np.array_equal(G.Apply(x), F.Apply(x))
    a2, _ = patch_update(a, N, 5 if len(N) == 2 else 3, 10.0, seed=7)
    A2 = stencil.build_laplacian(a2)
    mod = stencil.modified_dofs(A, A2)
    F.Update(A2, mod)
    G.Update(A2, mod)
    assert np.array_equal(G.Solve(b.T), F.Solve(b.T))


def test_rejects_mismatched_or_corrupt_files(tmp_path):
    N = (63, 63)
    _, A, b = problem(2, N, seed=62)
    F = make(N, A)
    with pytest.raises(MFError) as ei:
        F.save(tmp_path / "early.mfgpu")
    assert ei.value.status == _lib.MFGPU_ERR_STATE
    F.Factor()
    path = tmp_path / "factor.mfgpu"
    F.save(path)
    _, A31, _ = problem(2, (31, 31), seed=62)
    for other in (make((31, 31), A31), make(N, A, precision=MFGPU_MIXED)):
        with pytest.raises(ValueError, match="does not match"):
            other.load(path)
    raw = bytearray(path.read_bytes())
    raw[len(raw) // 2] ^= 0x40              # one bit of the payload
    bad = tmp_path / "corrupt.mfgpu"
    bad.write_bytes(bytes(raw))
    G = make(N, A)
    with pytest.raises(ValueError, match="checksum"):
        G.load(bad)
    with pytest.raises(MFError) as ei:      # a failed load leaves the handle unfactored
        G.Solve(b[0])
    assert ei.value.status == _lib.MFGPU_ERR_STATE
    G.load(path)                            # the intact file still loads
    assert np.array_equal(G.Solve(b[0]), F.Solve(b[0]))
