"""The column-batched Arnoldi stability driver (chanflow.arnoldi_columns) on
the CPU, with the oracle's propagator matvec (PFC/arnoldi.f90:485-567) as the
operator: its 10 leading eigenvalues about laminar Poiseuille flow (16x17x16,
Re 2900, T = 0.5) equal the eigenvalues of the dense per-column operators
(built column by column from the same matvec) to 1e-12, with explicit
residuals below 1e-10."""
import numpy as np


class OracleOperator:
    """The oracle's linearized propagator behind the ChannelFlow matvec API."""

    def __init__(self, orc, cf, nx=16, ny=17, nz=16, dt=0.01):
        self.nx, self.ny, self.nz, self.dt = nx, ny, nz, dt
        grid = cf.Grid(nx, ny, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=1.5)
        self.o = orc.Oracle(nx, ny, nz, re=2900.0, dt=dt, stretch=1.5, fix_mass=0)
        self.o.baseflow[:, 0] = 1 - grid.yh ** 2

    def arnoldi_matvec(self, x, tend):
        return self.o.arnoldi_matvec(np.asarray(x).reshape((self.nx, self.nz, self.ny + 1, 3), order="F"), tend)

    def scalars(self):
        return {"dt": self.dt}


def test_column_arnoldi_matches_dense_column_spectra(cf, orc):
    ch = cf.chanflow
    op = OracleOperator(orc, cf)
    tend = 50
    mu, lam, res, cols = ch.arnoldi_columns(op, tend, ncv=30, nev=10, restarts=4)
    # dense operators of all columns at once: one matvec per basis vector
    C = ch.stability_columns(op.nx, op.nz)
    n = (op.ny + 1) * 3
    a, b = C[:, 0], C[:, 1]
    nx, nz = op.nx, op.nz

    def embed(V):
        Ch = np.zeros((nz, nx // 2 + 1, n), complex)
        Ch[b, a] = V
        k0 = a == 0
        Ch[(-b[k0]) % nz, 0] = np.conj(V[k0])
        X = np.fft.irfft2(Ch, s=(nz, nx), axes=(0, 1))
        return np.asfortranarray(X.transpose(1, 0, 2).reshape(nx, nz, op.ny + 1, 3, order="C"))

    def extract(X):
        Xz = np.ascontiguousarray(np.asarray(X).reshape(nx, nz, n, order="C").transpose(1, 0, 2))
        return np.fft.rfft2(Xz, axes=(0, 1))[b, a]

    M = np.zeros((len(C), n, n), complex)
    for i in range(n):
        V = np.zeros((len(C), n), complex)
        V[:, i] = 1
        M[:, :, i] = extract(op.arnoldi_matvec(embed(V), tend))
    ev = np.linalg.eigvals(M)
    top = np.sort(np.abs(ev).ravel())[::-1][:10]
    assert np.abs(np.abs(mu) - top).max() < 1e-12, (np.abs(mu), top)
    assert res.max() < 1e-10, res
    # lam = log(mu)/T
    assert np.allclose(np.exp(lam * tend * op.dt), mu, rtol=1e-12)
