"""CPU restatement of the LES mode's subgrid stresses -- TEST INFRASTRUCTURE
ONLY: the checker of csrc/les.cuh and of the flux kernel's subgrid-stress
mode.  The reference has no subgrid model code (its subgrid = 1 branch,
PFC/main_mpi.f90:74-78, calls modules that are not in the repository), so
this restates the model the product defines:

- physical planes u, v, w of every y plane on the dealiased grid by the
  oracle's own xz_fft_complex_to_real (PFC/transform.f90:339-409);
- at interior yh planes k = 2..ny the resolved gradient G_ij = du_i/dx_j:
  central differences in x and z on the dealiased grid; du/dy, dw/dy over
  yh(k-1)..yh(k+1); dv/dy = dh(k) (v(k) - v(k-1)); v at yh(k) the mean of its
  two y planes;
- eddy viscosity: tau = -2 nu_t S^d, nu_t = (cs Delta (1 - exp(-y+/A+)))^2
  |S|, Delta = (lx/nx dy lz/nz)^(1/3), y+ = (1 - |yh|) u_tau Re, u_tau^2 =
  the mean of |dU/dy| at the two walls over Re;
- the stresses enter the momentum fluxes at the points of the products
  (PFC/pass1.f90:134-226): u and w equations tau_i1, tau_i3 on plane k and
  tau_i2 on the y planes as half sums (zero on the walls), v equation
  iu-weighted tau_12, tau_23 and tau_22 on the yh planes around it; the
  divergence is the oracle's parallel_divergence_of_fluxes
  (PFC/transform.f90:573-690), linear in its inputs, so the LES nonlinear
  term is the oracle's plus the divergence of the stress fluxes.
"""
import numpy as np


def physical_planes(o):
    """(ny+1, 3, nz2, nx2) physical velocity of the oracle's data1."""
    d1 = o.data1
    ny1 = o.ny + 1
    P = np.zeros((ny1, 3, o.nz2, o.nx2))
    for pl in range(ny1):
        for c in range(3):
            P[pl, c] = o.xz_c2r(d1[:, :, pl, c]).T
    return P


def gradient(P, o, k, lx, lz):
    """G[i, j] (3, 3, nz2, nx2) at yh plane k (1-based)."""
    y, yh, dh = o.grid("y"), o.grid("yh"), o.grid("dh")
    hx, hz = lx / o.nx2, lz / o.nz2
    Pm, P0, Pp = P[k - 2], P[k - 1], P[k]

    def ddx(f):
        return (np.roll(f, -1, axis=1) - np.roll(f, 1, axis=1)) / (2 * hx)

    def ddz(f):
        return (np.roll(f, -1, axis=0) - np.roll(f, 1, axis=0)) / (2 * hz)

    vc = 0.5 * (Pm[1] + P0[1])
    idy = 1.0 / (yh[k] - yh[k - 2])
    G = np.empty((3, 3) + P0[0].shape)
    G[0] = ddx(P0[0]), (Pp[0] - Pm[0]) * idy, ddz(P0[0])
    G[1] = ddx(vc), (P0[1] - Pm[1]) * dh[k - 1], ddz(vc)
    G[2] = ddx(P0[2]), (Pp[2] - Pm[2]) * idy, ddz(P0[2])
    return G


def strain_nut(G, o, k, re, lx, lz, cs, aplus, d_um_dy):
    """Trace-free strain (11, 22, 33, 12, 13, 23) and nu_t at plane k."""
    y, yh = o.grid("y"), o.grid("yh")
    tr = (G[0, 0] + G[1, 1] + G[2, 2]) / 3.0
    Sd = np.array([G[0, 0] - tr, G[1, 1] - tr, G[2, 2] - tr, 0.5 * (G[0, 1] + G[1, 0]),
                   0.5 * (G[0, 2] + G[2, 0]), 0.5 * (G[1, 2] + G[2, 1])])
    ss = Sd[0] ** 2 + Sd[1] ** 2 + Sd[2] ** 2 + 2 * (Sd[3] ** 2 + Sd[4] ** 2 + Sd[5] ** 2)
    smag = np.sqrt(2 * ss)
    delta = np.cbrt(lx / o.nx * (y[k - 1] - y[k - 2]) * lz / o.nz)
    utau = np.sqrt(0.5 * (abs(d_um_dy[0]) + abs(d_um_dy[-1])) / re)
    yplus = (1 - abs(yh[k - 1])) * utau * re
    f = cs * delta * (1 - np.exp(-yplus / aplus))
    return Sd, f * f * smag


def eddy_viscosity_stresses(o, re, lx, lz, cs=0.1, aplus=25.0, P=None):
    """S (ny+1, 6, nz2, nx2): the eddy-viscosity stresses on the yh planes
    (components 11, 22, 33, 12, 13, 23; zero on the wall planes)."""
    P = physical_planes(o) if P is None else P
    S = np.zeros((o.ny + 1, 6, o.nz2, o.nx2))
    dud = o.d_um_dy.copy()
    for k in range(2, o.ny + 1):
        G = gradient(P, o, k, lx, lz)
        Sd, nut = strain_nut(G, o, k, re, lx, lz, cs, aplus, dud)
        S[k - 1] = -2 * nut * Sd
    return S


def stress_divergence(o, S):
    """The divergence of the stress fluxes in data1 layout (nz, nx/2+1,
    ny+1, 3), added to the nonlinear term by the LES mode."""
    ny = o.ny
    dh, dn, iu = o.grid("dh"), o.grid("dn"), o.grid("iu")
    out = np.zeros((o.nz, o.nxh, ny + 1, 3), dtype=np.complex128, order="F")
    T = lambda pl, c: S[pl, c].T          # (nx2, nz2) Fortran order for the oracle
    zero = np.zeros((o.nx2, o.nz2))
    for k in range(2, ny + 1):
        up = k < ny
        # u and w equations at yh plane k
        for eq, (cx, cy, cz) in ((0, (0, 3, 4)), (2, (4, 5, 2))):
            fy1 = 0.5 * (T(k - 1, cy) + T(k, cy)) if up else zero
            fy0 = 0.5 * (T(k - 2, cy) + T(k - 1, cy)) if k > 2 else zero
            out[:, :, k - 1, eq] = o.div_fluxes(T(k - 1, cx), dh[k - 1] * (fy1 - fy0), T(k - 1, cz))
        # v equation at y plane k (k <= ny-1)
        if k <= ny - 1:
            i1, i2 = iu[0, k - 1], iu[1, k - 1]
            xf = i1 * T(k - 1, 3) + i2 * T(k, 3)
            zf = i1 * T(k - 1, 5) + i2 * T(k, 5)
            out[:, :, k - 1, 1] = o.div_fluxes(xf, dn[k - 1] * (T(k, 1) - T(k - 1, 1)), zf)
    return out
