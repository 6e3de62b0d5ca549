"""GPU: the update-serving loop (mfgpu_server_*).

Every request's answer must equal (to 1e-12 in FP64, 1e-10 residual in mixed)
the solve of a fresh factorization of the base matrix under that request's
change alone, be bit-identical whether the request runs alone or batched with
others in flight (their root paths factored by the same launches), and leave
the base factorization untouched.
"""
import numpy as np
import pytest

from mfgpu import MF2D, MF3D, MFGPU_MIXED, MFError, Server, stencil
from problems import rel

pytestmark = pytest.mark.gpu


def base_problem(N, seed):
    a = stencil.loguniform_coefficients(N, 0.1, 10.0, seed)
    return a, stencil.build_laplacian(a)


def make(N, A, **kw):
    return MF2D(A, N[0], N[1], 1, 4, **kw) if len(N) == 2 else MF3D(A, N[0], N[1], N[2], 1, 4, **kw)


def requests(N, count, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        side = int(rng.integers(3, 10))
        lo = [int(rng.integers(0, n - side + 1)) for n in N]
        factor = float(0.1 * 100.0 ** rng.random())
        k = int(rng.integers(1, 4))
        b = rng.uniform(-1, 1, size=(int(np.prod(N)), k))
        out.append((lo, [l + side for l in lo], factor, b))
    return out


@pytest.mark.parametrize("N,precision", [((127, 127), None), ((63, 63), MFGPU_MIXED),
                                         ((15, 15, 15), None)])
def test_serving_alone_equals_mixed_and_fresh_factorization(N, precision):
    kw = {} if precision is None else {"precision": precision}
    a, A = base_problem(N, 91)
    F = make(N, A, **kw)
    F.Factor()
    b0 = np.random.Generator(np.random.PCG64(3)).uniform(-1, 1, A.n)
    x0 = F.Solve(b0)
    reqs = requests(N, 6, 17)
    S = Server(F, a, slots=3, pool_gb=2.0)
    alone = []
    for lo, hi, f, b in reqs:              # one at a time
        alone.append(S.wait(S.submit(lo, hi, f, b))[0])
    tickets = [S.submit(lo, hi, f, b) for lo, hi, f, b in reqs]   # all in flight
    mixed = [S.wait(t) for t in tickets]
    # requests in flight together were served in shared batches (one set of
    # level launches for all their root paths)
    assert max(info["batch"] for _, info in mixed) >= 2
    for (lo, hi, f, b), xa, (xm, info) in zip(reqs, alone, mixed):
        assert info["status"] == 0 and info["fronts"] > 0
        assert np.array_equal(xa, xm)       # the same alone and in the mix
        ar = stencil.scale_box(a, lo, hi[0] - lo[0], f)
        Ar = stencil.build_laplacian(ar)
        if precision is None:
            G = make(N, Ar)
            G.Factor()
            assert rel(xm, G.Solve(b)) < 1e-12
        else:
            assert info["residual"] <= 1e-10
            for c in range(b.shape[1]):
                assert np.linalg.norm(Ar.matvec(xm[:, c]) - b[:, c]) / np.linalg.norm(b[:, c]) <= 2e-10
    S.close()
    assert np.array_equal(F.Solve(b0), x0)   # the base factorization is untouched


def test_serving_rejects_requests_larger_than_the_pool():
    N = (127, 127)
    a, A = base_problem(N, 92)
    F = make(N, A)
    F.Factor()
    S = Server(F, a, slots=1, pool_gb=1.0 / 1024)     # 1 MiB: smaller than any root path
    t = S.submit([5, 5], [9, 9], 2.0, np.ones(A.n))
    with pytest.raises(MFError) as ei:
        S.wait(t)
    assert ei.value.status == 4
    S.close()
