"""One-time BEM solve on the GPU (AxisymmetricBEMSolution.solve,
bem/axisymmetric.py:411-443): the collocation matrix is assembled by the
CUDA kernel behind spt_bem_assemble (adaptive bisection + Gauss-4 per
leaf, one thread per node-segment pair) and the dense system is solved by
LU (torch.linalg.solve -> cuSOLVER), all in float64."""

import ctypes

import numpy as np

from . import _lib


def assemble(profile, refine_ratio=1.0, max_depth=20, device="cuda"):
    import torch

    prof = np.asarray(profile, dtype=np.float64)
    n = len(prof)
    d = torch.device(device)
    pr = torch.as_tensor(np.ascontiguousarray(prof[:, 0]), device=d)
    pz = torch.as_tensor(np.ascontiguousarray(prof[:, 1]), device=d)
    gx, gw = np.polynomial.legendre.leggauss(4)
    gx = torch.as_tensor(gx, device=d)
    gw = torch.as_tensor(gw, device=d)
    A = torch.empty((n, n), dtype=torch.float64, device=d)
    stream = torch.cuda.current_stream(d)
    _lib.check(_lib.lib().spt_bem_assemble(pr.data_ptr(), pz.data_ptr(), n, float(refine_ratio), int(max_depth),
                                           gx.data_ptr(), gw.data_ptr(), A.data_ptr(),
                                           ctypes.c_void_p(stream.cuda_stream)), "spt_bem_assemble")
    return A


def solve_dirichlet(profile, dirichlet_fn, refine_ratio=1.0, max_depth=20, device="cuda"):
    """Nodal density sigma with S[sigma](node_i) = dirichlet_fn(rho_i, z_i)."""
    import torch

    prof = np.asarray(profile, dtype=np.float64)
    A = assemble(prof, refine_ratio, max_depth, device)
    b = torch.as_tensor(np.array([dirichlet_fn(r, z) for r, z in prof], dtype=np.float64), device=A.device)
    return torch.linalg.solve(A, b).cpu().numpy()
