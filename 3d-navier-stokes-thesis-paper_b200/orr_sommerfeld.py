"""Orr-Sommerfeld eigenmodes of plane Poiseuille flow, and the efn.m file the
reference's which_test 2/5/8 runs read.

The reference's Orr-Sommerfeld test (PFC/init_vel.f90:95-159) starts from the
least-stable two-dimensional mode at Re = 7500, alpha = 1 (lx = 2 pi), whose
eigenfunction it reads from efn.m: 4 x 65 numbers, one per line -- Re u,
Im u, Re v, Im v at the 65 Chebyshev-Gauss-Lobatto points y_j = cos(pi j/64),
j = 0..64 (READ_EIGENFUNCTION, PFC/init_vel.f90:540-640).  That file was made
outside the reference (a MATLAB Chebyshev code) and is not shipped; this
module makes it.  The reference fixes the mode's phase speed at 0.24989154
(PFC/setup.f90:1386-1388, the dt of a two-period run).

Method: Chebyshev collocation of the Orr-Sommerfeld equation for
v = phi(y) exp(i alpha (x - c t)),

    (U - c)(phi'' - a^2 phi) - U'' phi = (phi'''' - 2 a^2 phi'' + a^4 phi) / (i a Re),

U = 1 - y^2, phi(+-1) = phi'(+-1) = 0, as the generalised eigenproblem
A phi = lambda B phi with lambda = -i alpha c (time dependence exp(lambda t)),
B = D2 - a^2, A = (D4 - 2 a^2 D2 + a^4)/Re - i a U (D2 - a^2) + i a U''.
The clamped fourth derivative is the collocation derivative of
phi = (1 - y^2) q (Trefethen, Spectral Methods in MATLAB, 2000, program 40).
Streamwise velocity from continuity: u = i phi' / alpha.
"""
import numpy as np

NCHEB = 65                 # READ_EIGENFUNCTION's NCHEB
PHASE_SPEED_RE7500 = 0.24989154   # PFC/setup.f90:1387


def cheb(n):
    """Chebyshev-Gauss-Lobatto points x_j = cos(pi j / n), j = 0..n, and the
    collocation differentiation matrix (Trefethen's cheb)."""
    x = np.cos(np.pi * np.arange(n + 1) / n)
    c = np.ones(n + 1)
    c[0] = c[-1] = 2.0
    c *= (-1.0) ** np.arange(n + 1)
    dx = x[:, None] - x[None, :]
    d = np.outer(c, 1.0 / c) / (dx + np.eye(n + 1))
    d -= np.diag(d.sum(axis=1))
    return d, x


def os_modes(re, alpha, n=NCHEB - 1):
    """All Orr-Sommerfeld eigenvalues lambda (= -i alpha c) and eigenvectors
    phi on the n - 1 interior collocation points, for plane Poiseuille flow."""
    import scipy.linalg as sl
    d, x = cheb(n)
    d2 = d @ d
    s = np.diag(np.r_[0.0, 1.0 / (1.0 - x[1:n] ** 2), 0.0])
    d4 = (np.diag(1.0 - x ** 2) @ np.linalg.matrix_power(d, 4)
          - 8.0 * np.diag(x) @ np.linalg.matrix_power(d, 3) - 12.0 * d2) @ s
    d2i, d4i = d2[1:n, 1:n], d4[1:n, 1:n]
    eye = np.eye(n - 1)
    u = np.diag(1.0 - x[1:n] ** 2)
    a2 = alpha * alpha
    a = (d4i - 2.0 * a2 * d2i + a2 * a2 * eye) / re - 1j * alpha * u @ (d2i - a2 * eye) - 2j * alpha * eye
    b = d2i - a2 * eye
    lam, vec = sl.eig(a, b)
    return lam, vec, d, x


def least_stable(re=7500.0, alpha=1.0, n=NCHEB - 1):
    """The least-stable mode: (c, u, v, x) with c the complex phase speed
    (growth rate alpha * c.imag), u and v at the n + 1 collocation points
    x_j = cos(pi j / n), normalised to max |u| = 1 with u real and positive
    where |u| peaks."""
    lam, vec, d, x = os_modes(re, alpha, n)
    ok = np.isfinite(lam)
    k = np.flatnonzero(ok)[np.argmax(lam[ok].real)]
    c = 1j * lam[k] / alpha
    phi = np.zeros(n + 1, complex)
    phi[1:n] = vec[:, k]
    u = 1j * (d @ phi) / alpha
    j = np.argmax(np.abs(u))
    scale = 1.0 / u[j]
    return c, u * scale, phi * scale, x


def efn_columns(u, v):
    """The (65, 4) array efn.m holds: Re u, Im u, Re v, Im v."""
    return np.stack([u.real, u.imag, v.real, v.imag], axis=1)


def write_efn(path, re=7500.0, alpha=1.0):
    """Write efn.m for the reference's which_test 2 (and 5, 8: the same
    two-dimensional mode, rotated by the run's beta): 260 numbers, one per
    line, column after column.  Returns the phase speed c."""
    c, u, v, _ = least_stable(re, alpha)
    cols = efn_columns(u, v)
    with open(path, "w") as f:
        for k in range(4):
            for j in range(NCHEB):
                f.write(f"{cols[j, k]: .17e}\n")
    return c


def mode_energy(data1, dyh, x=1, z=0):
    """The kinetic energy of Fourier column (kz index z, kx index x) of a
    velocity field in data1 layout (nz, nx/2+1, ny+1, 3), integrated over y
    with dyh as rhs_solve does for ke(x,z) (PFC/pass2.f90:113-117): |u|^2 +
    |w|^2 on the yh planes and |v|^2 averaged onto them."""
    cu = data1[z, x]
    ny = cu.shape[0] - 1
    t = np.abs(cu[:, 0]) ** 2 + np.abs(cu[:, 2]) ** 2
    t[0] += np.abs(cu[0, 1]) ** 2
    t[1:ny] += np.abs(0.5 * (cu[1:ny, 1] + cu[0:ny - 1, 1])) ** 2
    t[ny] += np.abs(cu[ny - 1, 1]) ** 2
    return float(np.sum(dyh * t))
