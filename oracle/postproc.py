"""CPU restatement of the post-processing arithmetic, as test infrastructure
(only the tests call it): the velocity on the output grid of the VTK
snapshot (PFC/read_write.f90:433-462 with yskip = 1), the velocity-gradient
tensor, vorticity, Q-criterion and the discriminant of the ParaView
Calculator (ParaView-Code/DiscriminantFilter.cpd:17), and the per-plane
moments of PFC/stats.f90:423-456 for one snapshot.  Inverse transforms are
the oracle's small_fft_complex_to_real; y derivatives the 3-point Lagrange
stencils of stats.f90's setup_diff (PFC/stats.f90:66-70).  FP64, numpy."""
import numpy as np


def yh_plane(d1, c, pl, ny):
    """Spectral plane (nz, nx/2+1) of component c on yh(pl) (0-based)."""
    if c != 1:
        return d1[:, :, pl, c]
    if pl == 0:
        return d1[:, :, 0, 1]
    if pl == ny:
        return d1[:, :, ny - 1, 1]
    return 0.5 * (d1[:, :, pl - 1, 1] + d1[:, :, pl, 1])


def lagrange_first(yh):
    n1 = len(yh)
    w = np.zeros((n1, 3))
    s = np.zeros((n1, 3), int)
    for j in range(n1):
        a = 0 if j == 0 else (n1 - 3 if j == n1 - 1 else j - 1)
        nd = [a, a + 1, a + 2]
        for q in range(3):
            xq, xr, xs = yh[nd[q]], yh[nd[(q + 1) % 3]], yh[nd[(q + 2) % 3]]
            w[j, q] = ((yh[j] - xr) + (yh[j] - xs)) / ((xq - xr) * (xq - xs))
            s[j, q] = nd[q]
    return w, s


def velocity_and_gradient(o, d1, yh, kx, kz):
    """u (nx, n1, nz, 3) and A (nx, n1, nz, 3, 3), A[..., i, j] = du_i/dx_j."""
    nz, nxh, n1, _ = d1.shape
    ny = n1 - 1
    nx = 2 * (nxh - 1)
    w, s = lagrange_first(yh)
    KX = np.broadcast_to(kx[None, :], (nz, nxh))
    KZ = np.broadcast_to(kz[:, None], (nz, nxh))
    u = np.zeros((nx, n1, nz, 3))
    A = np.zeros((nx, n1, nz, 3, 3))
    c2r = lambda p: o.small_c2r(np.asfortranarray(p))
    for pl in range(n1):
        for c in range(3):
            p = yh_plane(d1, c, pl, ny)
            u[:, pl, :, c] = c2r(p)
            A[:, pl, :, c, 0] = c2r(1j * KX * p)
            A[:, pl, :, c, 2] = c2r(1j * KZ * p)
            dy = sum(w[pl, q] * yh_plane(d1, c, s[pl, q], ny) for q in range(3))
            A[:, pl, :, c, 1] = c2r(dy)
    return u, A


def invariants(A):
    """vorticity (..., 3), Q = -tr(A^2)/2, D = (6 tr(A^3)^2 - tr(A^2)^3)/8"""
    vort = np.stack([A[..., 2, 1] - A[..., 1, 2], A[..., 0, 2] - A[..., 2, 0], A[..., 1, 0] - A[..., 0, 1]], -1)
    A2 = np.einsum("...ij,...jk->...ik", A, A)
    tr2 = np.trace(A2, axis1=-2, axis2=-1)
    tr3 = np.einsum("...ij,...ji->...", A2, A)
    return vort, -0.5 * tr2, 0.125 * (6 * tr3 ** 2 - tr2 ** 3)


def plane_moments(u, vort):
    """(n1, 27): stats.f90's compute_velocity_moments and
    compute_vorticity_moments for one snapshot, normalised as at :258-268."""
    eps = np.finfo(np.float64).eps
    nx, n1, nz, _ = u.shape
    out = np.zeros((n1, 27))
    for j in range(n1):
        uu = u[:, j, :, :].reshape(-1, 3)
        ww = vort[:, j, :, :].reshape(-1, 3)
        for base, f, flux in ((0, uu, True), (15, ww, False)):
            m = f.mean(0)
            d = f - m
            var = (d ** 2).mean(0)
            out[j, base:base + 3] = m
            out[j, base + 3:base + 6] = var
            out[j, base + 6:base + 9] = (d ** 3).mean(0) / (var ** 1.5 + eps)
            out[j, base + 9:base + 12] = (d ** 4).mean(0) / (var ** 2 + eps)
            if flux:
                out[j, 12:15] = (d * d[:, 1:2]).mean(0)
    return out
