"""CPU restatement of init_buffer (PFC/init_jet_buffer.f90:358-483), as test
infrastructure: the fringe profile on the nx x nz grid, its small forward
transform and the dealiased inverse onto nx2 x nz2 (the oracle's
small_fft_real_to_complex and xz_fft_complex_to_real), times fringe_gain,
and the closed channel's target_inflow.  FP64, numpy."""
import numpy as np


def fringe_region(t, ts, tr, tf, te):
    """define_fringe_region, PFC/init_jet_buffer.f90:453-482"""
    f = np.zeros_like(t)
    f2 = np.zeros_like(t)
    for i, ti in enumerate(t):
        if ti > ts:
            if ti < tr:
                t2 = (ti - ts) / (tr - ts)
                f[i] = 1 / (1 + np.exp(1 / t2 + 1 / (t2 - 1)))
                f2[i] = t2
            elif tf < ti < te:
                t2 = (te - ti) / (te - tf)
                f[i] = 1 / (1 + np.exp(1 / t2 + 1 / (t2 - 1)))
                f2[i] = t2
            elif ti >= te:
                f[i] = 0.0
            else:
                f[i] = 1.0
    return f, f2


def init_buffer(o, nx, nz, lx, lz, yh, beta, fringe_gain, xfringe, zfringe, frac_xbuff, buff_xrise, buff_xfall,
                frac_zbuff):
    tx = np.arange(nx) * lx / nx
    tz = np.arange(nz) * lz / nz
    if xfringe == 1:
        xs = lx * (1 - frac_xbuff)
        fx, fx2 = fringe_region(tx, xs, xs + lx * buff_xrise, lx - lx * buff_xfall, lx)
    else:
        fx, fx2 = np.zeros(nx), np.zeros(nx)
    if zfringe == 1:
        fa, fa2 = fringe_region(tz, -1.0, -1.0, 0.0, frac_zbuff * lz)
        fb, fb2 = fringe_region(tz, lz - frac_zbuff * lz, lz, lz + 1, lz + 1)
        fz, fz2 = fa + fb, fa2 + fb2
    else:
        fz, fz2 = np.zeros(nz), np.zeros(nz)
    temp = np.zeros((nx, nz))
    for z in range(nz):
        for x in range(nx):
            if fx[x] < 1 and fz[z] < 1 and fx[x] * fz[z] > 0:
                t = np.sqrt(fx2[x] ** 2 + fz2[z] ** 2)
                temp[x, z] = 1 / (1 + np.exp(1 / t + 1 / (t - 1))) if t < 1 else 1.0
            else:
                temp[x, z] = max(fx[x], fz[z])
    buffer = fringe_gain * o.xz_c2r(o.small_r2c(np.asfortranarray(temp)))
    prof = 0.75 * (1 - np.asarray(yh) ** 8)
    target = np.zeros((len(yh), 3), order="F")
    target[:, 0] = prof * np.cos(beta)
    target[:, 2] = prof * np.sin(beta)
    return buffer, target
