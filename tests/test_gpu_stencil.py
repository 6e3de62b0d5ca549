"""GPU: stencil assembly and modified-DOF detection on the device.

The device values must equal the fixture's Laplacian (stencil.build_laplacian,
itself pinned bit for bit to test_include/DE/buildLaplacian.hpp) bit for bit,
and the modified DOFs of a coefficient box change must equal the host diff the
reference's test uses (test_src/DE/testMF2D.cpp:143-150).
"""
import numpy as np
import pytest
import torch

from mfgpu import MF2D, MF3D, stencil
from problems import rel

pytestmark = pytest.mark.gpu


def make(N, A):
    return MF2D(A, N[0], N[1], 1, 4) if len(N) == 2 else MF3D(A, N[0], N[1], N[2], 1, 4)


@pytest.mark.parametrize("N,h", [((31, 31), (1.0, 1.0, 1.0)), ((23, 57), (0.5, 0.25, 1.0)),
                                 ((15, 15, 15), (1.0, 1.0, 1.0)),
                                 ((13, 17, 11), (1 / 14, 1 / 18, 1 / 12))])
def test_device_assembly_bitwise(N, h):
    a = stencil.loguniform_coefficients(N, 0.1, 10.0, 77)
    A = stencil.build_laplacian(a, h=h[:len(N)])
    F = make(N, A)
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dv = torch.full((A.nnz,), np.nan, dtype=torch.float64, device="cuda")
    F.stencil_assemble_device(da.data_ptr(), dv.data_ptr(), h)
    assert np.array_equal(dv.cpu().numpy(), A.val)


@pytest.mark.parametrize("N,lo,side", [((63, 63), (5, 9), 9), ((63, 63), (0, 0), 4),
                                       ((63, 63), (58, 60), 9), ((23, 23, 23), (3, 4, 5), 4),
                                       ((23, 23, 23), (20, 0, 19), 5)])
def test_device_update_and_modified_dofs(N, lo, side):
    a1 = stencil.loguniform_coefficients(N, 0.1, 10.0, 78)
    a2 = stencil.scale_box(a1, lo, side, 10.0)
    A1, A2 = stencil.build_laplacian(a1), stencil.build_laplacian(a2)
    F = make(N, A1)
    F.Factor()
    b = np.random.Generator(np.random.PCG64(5)).uniform(-1, 1, A1.n)
    dv = torch.from_numpy(A1.val.copy()).cuda()
    da2 = torch.from_numpy(np.ascontiguousarray(a2)).cuda()
    hi = [min(l + side, n) for l, n in zip(lo, N)]
    mod = F.stencil_update_device(da2.data_ptr(), lo, hi, dv.data_ptr())
    assert np.array_equal(mod, stencil.modified_dofs(A1, A2))
    assert np.array_equal(dv.cpu().numpy(), A2.val)
    # and the device-built update drives the localized refactorization
    F.update_device(dv.data_ptr(), A1.nnz, mod)
    G = make(N, A2)
    G.Factor()
    assert rel(F.Solve(b), G.Solve(b)) < 1e-13
