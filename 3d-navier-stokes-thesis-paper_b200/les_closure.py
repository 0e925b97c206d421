"""The learned subgrid-stress closure of the LES mode: training data from
box-filtered DNS snapshots of this GPU solver, training on the GPU with the
tensor-core kernels (Mlp), and the a-priori and a-posteriori comparisons with
the eddy-viscosity closure and the filtered DNS.

The reference runs LES through its subgrid = 1 branch (PFC/main_mpi.f90:74-78)
with model modules that are not in the repository; its filter and statistics
helpers are PFC/setup.f90:814-889 and PFC/stats.f90:120-128,244-251.  This
module defines the learned closure the product uses:

- filtered DNS: the DNS velocity on its nx x nz grid (the small inverse
  transforms, PFC/transform.f90:950-1000), a centred box filter of `factor`
  points in x and z (the LES grid is nx/factor x nz/factor), v averaged onto
  the yh planes, tau_ij = filt(u_i u_j) - filt(u_i) filt(u_j) on the DNS yh
  planes, everything interpolated linearly in y to the LES planes;
- features: the LES context's own feature kernel (cfg_les_features) run on
  the filtered velocity loaded as an LES state, so that training and the
  LES see the same discrete gradients; points of the dealiased LES grid that
  coincide with LES grid points ((3m, 3n) <-> (2m, 2n) for the 3/2 rule);
- normalisation: each feature and target standardised by its mean and
  standard deviation over the training set;
- targets in the lower half-channel's frame (tau_12, tau_23 change sign for
  yh > 0), as the features are.
"""
import math

import numpy as np

from .chanflow import MIXED, ChannelFlow, Grid, Mlp

PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))   # 11, 22, 33, 12, 13, 23


def physical(data1, nx, nz):
    """(ny+1, 3, nz, nx) physical velocity of a data1 array (nz, nx/2+1,
    ny+1, 3) on the nx x nz grid: the unnormalised inverse sums."""
    a = np.moveaxis(np.asarray(data1), (2, 3), (0, 1))
    return np.fft.irfft(np.fft.ifft(a, axis=2, norm="forward"), n=nx, axis=3, norm="forward")


def spectral(phys):
    """Inverse of physical(): (ny+1, 3, nz, nx) -> data1 (nz, nx/2+1, ny+1, 3)."""
    c = np.fft.fft(np.fft.rfft(phys, axis=3, norm="forward"), axis=2, norm="forward")
    return np.asfortranarray(np.moveaxis(c, (0, 1), (2, 3)))


def box(f, r):
    """Centred box filter of r (odd) points in the last two axes, sampled at
    every r-th point: (..., nz, nx) -> (..., nz/r, nx/r)."""
    h = r // 2
    g = np.roll(np.roll(f, h, axis=-1), h, axis=-2)
    s = g.shape
    return g.reshape(s[:-2] + (s[-2] // r, r, s[-1] // r, r)).mean(axis=(-3, -1))


def interp_planes(f, yfrom, yto):
    """Linear interpolation along axis 0 from the points yfrom to yto."""
    i = np.clip(np.searchsorted(yfrom, yto) - 1, 0, len(yfrom) - 2)
    w = (yto - yfrom[i]) / (yfrom[i + 1] - yfrom[i])
    w = w.reshape((-1,) + (1,) * (f.ndim - 1))
    return (1 - w) * f[i] + w * f[i + 1]


def filter_snapshot(data1, gd, gl, factor=3):
    """Filtered DNS of one snapshot for the LES grid gl.  Returns the LES
    state data1 (nz, nx/2+1, ny+1, 3) of the filtered velocity and the
    stresses tau (ny_les-1, 6, nz, nx) on the LES yh planes 2..ny and the LES
    x-z grid, in the lower half-channel's frame."""
    ph = physical(data1, gd.nx, gd.nz)                    # (ny+1, 3, nz, nx)
    nyd = gd.ny
    u, w = ph[:, 0], ph[:, 2]
    vy = ph[:nyd, 1]                                      # v on y planes 1..ny
    vc = np.zeros_like(u)                                 # v on the yh planes
    vc[1:nyd] = 0.5 * (vy[:-1] + vy[1:])
    vel = (u, vc, w)
    fu = [box(q, factor) for q in vel]
    fv_y = box(vy, factor)
    tau = np.empty((nyd + 1, 6) + fu[0].shape[1:])
    for c, (i, j) in enumerate(PAIRS):
        tau[:, c] = box(vel[i] * vel[j], factor) - fu[i] * fu[j]
    tau[0] = tau[nyd] = 0.0
    # to the LES planes
    yhl, yl = gl.yh, gl.y
    st = np.zeros((gl.ny + 1, 3) + fu[0].shape[1:])
    st[:, 0] = interp_planes(fu[0], gd.yh, yhl)
    st[:, 2] = interp_planes(fu[2], gd.yh, yhl)
    st[:gl.ny, 1] = interp_planes(fv_y, gd.y, yl)
    st[0, 0] = st[gl.ny, 0] = st[0, 2] = st[gl.ny, 2] = 0.0   # no-slip walls
    st[0, 1] = st[gl.ny - 1, 1] = 0.0
    t = interp_planes(tau, gd.yh, yhl[1:gl.ny])
    up = yhl[1:gl.ny] > 0
    t[up, 3] *= -1
    t[up, 5] *= -1
    return spectral(st), t


class FeatureProbe:
    """An LES context used to compute the closure's features of given LES
    states (cfg_les_features) and the eddy-viscosity stresses there."""

    def __init__(self, gl, re, device=0, cs=0.1, aplus=25.0):
        import torch
        self.gl, self.torch = gl, torch
        self.flow = ChannelFlow(gl, re=re, dt=0.005, fix_mass=1, precision=MIXED, device=device)
        self.net = Mlp(device)              # unused weights: features only
        self.flow.set_les(2, cs=cs, aplus=aplus, mlp=self.net)
        self.n = (gl.ny - 1) * gl.nz2 * gl.nx2
        self.F = torch.zeros(self.n * 10, dtype=torch.float32, device=f"cuda:{device}")

    def features(self, data1, d_um_dy):
        """Features (ny-1, nz/2, nx/2, 10) and eddy-viscosity stresses
        (ny-1, 6, nz/2, nx/2) at the LES grid points (2m, 2n) of the state."""
        gl = self.gl
        self.flow.upload_state(data1, None, None)
        sc = self.flow.scalars()
        self.flow.set_scalars(sc["t_total"], sc["dt"], sc["p_grad"], d_um_dy)
        self.flow.les_features(self.F.data_ptr())
        F = self.F.cpu().numpy().reshape(gl.ny - 1, gl.nz2, gl.nx2, 10)[:, ::3, ::3]
        S = self.flow.les_stresses()[1:gl.ny, :, ::3, ::3]
        up = gl.yh[1:gl.ny] > 0
        S[up, 3] *= -1
        S[up, 5] *= -1
        return F, S

    def close(self):
        self.flow.close()
        self.net.close()


def wall_gradient(data1, g):
    """d_um_dy at the two walls (the mean-flow wall gradient of
    PFC/init_vel.f90:332-341) as an (ny,) array with the end values set."""
    u = np.real(data1[0, 0, :, 0])
    d = np.zeros(g.ny)
    d[0] = g.dm[0, 0] * u[0] + g.dm[1, 0] * u[1] + g.dm[2, 0] * u[2]
    d[-1] = g.dm[0, 1] * u[g.ny - 2] + g.dm[1, 1] * u[g.ny - 1] + g.dm[2, 1] * u[g.ny]
    return d


def deviatoric(t):
    """(..., 6, ...) stress components along axis 1 minus one third of the trace."""
    t = t.copy()
    tr = (t[:, 0] + t[:, 1] + t[:, 2]) / 3.0
    for c in range(3):
        t[:, c] -= tr
    return t


def init_params(seed=0):
    """He-normal weights (standard deviation sqrt(2 / fan_in)) and zero
    biases in the network's flat parameter order (cfg_mlp_set_params)."""
    rng = np.random.default_rng(seed)
    parts = []
    for nout, nin in ((64, 10), (64, 64), (64, 64), (6, 64)):
        parts.append(rng.standard_normal(nout * nin) * math.sqrt(2.0 / nin))
        parts.append(np.zeros(nout))
    return np.concatenate(parts).astype(np.float32)


def train(X, T, device=0, iters=3000, batch=4096, lr=2e-3, seed=0, log_every=500):
    """Fit the network to normalised features X (n, 10) and targets T (n, 6)
    with Adam (cosine learning-rate decay) on the GPU.  Returns (net, losses)."""
    import torch
    dev = torch.device("cuda", device)
    xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
    td = torch.from_numpy(np.ascontiguousarray(T, dtype=np.float32)).to(dev)
    net = Mlp(device, init_params(seed))
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    losses = []
    n = xd.shape[0]
    for it in range(iters):
        idx = torch.randint(0, n, (batch,), device=dev, dtype=torch.int32, generator=gen)
        net.accumulate_grad(xd.data_ptr(), td.data_ptr(), idx.data_ptr(), batch)
        if it % log_every == 0 or it == iters - 1:
            losses.append((it, net.grads()[1]))
        net.adam_step(lr * 0.5 * (1 + math.cos(math.pi * it / iters)))
    torch.cuda.synchronize(dev)
    if net.status() != 0:
        raise RuntimeError("closure network: a tensor-core wait gave up")
    return net, losses


def predict(net, X, device=0):
    """Network outputs (n, 6) for normalised features X (n, 10)."""
    import torch
    dev = torch.device("cuda", device)
    xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
    yd = torch.empty((X.shape[0], 6), dtype=torch.float32, device=dev)
    net.forward(xd.data_ptr(), yd.data_ptr(), X.shape[0])
    return yd.cpu().numpy()


def profile_stats(data1, g):
    """Mean streamwise velocity on the yh planes and the resolved Reynolds
    stresses <u'u'>, <v'v'>, <w'w'>, <u'v'> (plane averages), from a state."""
    ph = physical(data1, g.nx, g.nz)
    u, w = ph[:, 0], ph[:, 2]
    vc = np.zeros_like(u)
    vc[1:g.ny] = 0.5 * (ph[:g.ny - 1, 1] + ph[1:g.ny, 1])
    U = u.mean(axis=(1, 2))
    up, vp, wp = u - U[:, None, None], vc - vc.mean(axis=(1, 2))[:, None, None], w - w.mean(axis=(1, 2))[:, None, None]
    return U, np.stack([(up * up).mean(axis=(1, 2)), (vp * vp).mean(axis=(1, 2)), (wp * wp).mean(axis=(1, 2)),
                        (up * vp).mean(axis=(1, 2))])


def _events(torch, flow):
    st = torch.cuda.ExternalStream(flow.stream_ptr())
    return st, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def advance_to(flow, t_end, chunk=10):
    """Steps in chunks until t_total reaches t_end (adaptive dt)."""
    n = 0
    while flow.scalars()["t_total"] < t_end - 1e-12:
        flow.timestep(chunk)
        n += chunk
    return n


def run_c4(nx=384, ny=193, nz=384, factor=3, re=10350.0, stretch=1.5, ampl=0.5, seed=4, spinup=60.0,
           nsnap=40, snap_dt=0.5, cfl=0.5, train_iters=3000, batch=4096, lr=2e-3, les_spin=20.0, les_avg=20.0,
           cs=0.1, beta=0.0, device=0, log=print, artifact=None):
    """Configuration C4 end to end: DNS from the turbulent-profile initial
    field (which_test 4 plus seeded noise) at nx x ny x nz, nsnap snapshots
    snap_dt apart after `spinup` time units, box-filtered by `factor` in x
    and z onto the LES grid (nx/factor) x ((ny-1)/factor+1) x (nz/factor);
    the closure trained on all snapshots but the last, judged a priori on the
    last against the eddy viscosity, and LES runs (no model, eddy viscosity,
    learned closure) from the first filtered snapshot against the filtered
    DNS mean profile and resolved Reynolds stresses.  All steps mixed
    precision with adaptive dt (cfl_max = cfl).  artifact: an .npz path where
    the a-posteriori inputs are saved (les_from_artifact reruns them).
    Returns a dict of results."""
    import time
    import torch
    out = {"config": dict(nx=nx, ny=ny, nz=nz, factor=factor, re=re, stretch=stretch, ampl=ampl, spinup=spinup,
                          nsnap=nsnap, snap_dt=snap_dt, cfl=cfl, train_iters=train_iters, les_spin=les_spin,
                          les_avg=les_avg, cs=cs, beta=beta)}
    lx, lz = 4 * np.pi, 2 * np.pi
    gd = Grid(nx, ny, nz, lx=lx, lz=lz, stretch=stretch)
    nyl = (ny - 1) // factor + 1
    gl = Grid(nx // factor, nyl, nz // factor, lx=lx, lz=lz, stretch=stretch)
    # DNS
    t0 = time.time()
    dns = ChannelFlow(gd, re=re, dt=0.002, fix_mass=1, dt_flag=1, cfl_max=cfl, precision=MIXED, device=device)
    dns.define_initial_field(4, seed=seed, ampl=ampl)
    st, e0, e1 = _events(torch, dns)
    e0.record(st)
    nsteps = advance_to(dns, spinup)
    e1.record(st)
    e1.synchronize()
    dns_ms = e0.elapsed_time(e1) / nsteps
    sc = dns.scalars()
    out["dns"] = {"spinup_steps": nsteps, "ms_per_step": dns_ms, "dt": sc["dt"], "status": dns.status(),
                  "ms_per_time_unit": e0.elapsed_time(e1) / sc["t_total"]}
    log(f"DNS spin-up: {nsteps} steps to t = {sc['t_total']:.2f}, {dns_ms:.3f} ms/step, dt {sc['dt']:.4g}")
    probe = FeatureProbe(gl, re, device=device, cs=cs)
    feats, targs, evs, states, retau = [], [], [], [], []
    Uf, Rf = 0.0, 0.0
    for s in range(nsnap):
        if s:
            advance_to(dns, dns.scalars()["t_total"] + snap_dt)
        d1 = dns.download_state()[0]
        les_d1, tau = filter_snapshot(d1, gd, gl, factor)
        F, S = probe.features(les_d1, wall_gradient(les_d1, gl))
        feats.append(F)
        targs.append(tau[:, :, ::2, ::2])
        evs.append(S)
        if s == 0:
            states.append(les_d1)
        U, R = profile_stats(les_d1, gl)
        Uf, Rf = Uf + U / nsnap, Rf + R / nsnap
        dud = dns.scalars()["d_um_dy"]
        retau.append(math.sqrt(0.5 * (abs(dud[0]) + abs(dud[-1])) / re) * re)
    out["dns"]["re_tau_snapshots"] = [round(v, 2) for v in retau]
    out["dns"]["status_end"] = dns.status()
    out["dns"]["t_end"] = dns.scalars()["t_total"]
    dns.close()
    probe.close()
    log(f"{nsnap} snapshots filtered ({time.time() - t0:.1f} s so far)")
    # training set: all snapshots but the last
    X = np.concatenate([f.reshape(-1, 10) for f in feats[:-1]])
    Tt = np.concatenate([np.moveaxis(t, 1, -1).reshape(-1, 6) for t in targs[:-1]])
    mi, si = X.mean(axis=0), X.std(axis=0) + 1e-12
    mo, so = Tt.mean(axis=0), Tt.std(axis=0) + 1e-30
    t1 = time.time()
    net, losses = train((X - mi) / si, (Tt - mo) / so, device=device, iters=train_iters, batch=batch, lr=lr)
    out["training"] = {"samples": int(X.shape[0]), "losses": losses, "s": time.time() - t1}
    log(f"trained on {X.shape[0]} samples: loss {losses[0][1]:.4f} -> {losses[-1][1]:.4f}")
    # a priori on the held-out snapshot (deviatoric parts, the part that moves the flow)
    Xh = feats[-1].reshape(-1, 10)
    th = np.moveaxis(targs[-1], 1, -1).reshape(-1, 6)
    pred = predict(net, (Xh - mi) / si, device) * so + mo
    ev = np.moveaxis(evs[-1], 1, -1).reshape(-1, 6)

    def dev_err(a):
        d, r = deviatoric(a[:, :, None]) - deviatoric(th[:, :, None]), deviatoric(th[:, :, None])
        return float(np.linalg.norm(d) / np.linalg.norm(r))

    def corr(a, c):
        return float(np.corrcoef(a[:, c], th[:, c])[0, 1])

    out["a_priori"] = {"nn_deviatoric_rel_err": dev_err(pred), "ev_deviatoric_rel_err": dev_err(ev),
                       "nn_corr_12": corr(pred, 3), "ev_corr_12": corr(ev, 3), "points": int(th.shape[0])}
    log(f"a priori: deviatoric error NN {out['a_priori']['nn_deviatoric_rel_err']:.3f}, "
        f"eddy viscosity {out['a_priori']['ev_deviatoric_rel_err']:.3f}")
    if artifact:
        # what the a-posteriori runs need, to rerun them without the DNS
        np.savez_compressed(artifact, state=states[0].astype(np.complex64), Uf=Uf, Rf=Rf, params=net.get_params(),
                            mi=mi, si=si, mo=mo,
                            so=so, grid=np.array([gl.nx, gl.ny, gl.nz]), stretch=stretch, re=re,
                            dns_ms_per_time_unit=out["dns"]["ms_per_time_unit"])
    out["les"] = les_runs(gl, re, states[0], Uf, Rf, net, (mi, si, mo, so), cfl, les_spin, les_avg, cs, beta,
                          device, log)
    out["speedup_per_time_unit"] = {k: out["dns"]["ms_per_time_unit"] / v["ms_per_time_unit"]
                                    for k, v in out["les"].items()}
    out["filtered_dns"] = {"U": Uf.tolist(), "uv": Rf[3].tolist()}
    net.close()
    return out


def les_runs(gl, re, state, Uf, Rf, net, norm, cfl=0.5, les_spin=20.0, les_avg=20.0, cs=0.1, beta=0.0, device=0,
             log=print, models=(("none", 0), ("eddy_viscosity", 1), ("learned", 2))):
    """LES on grid gl from the filtered state, one run per closure: les_spin
    time units, then statistics every 0.5 time units over les_avg, against
    the filtered DNS mean profile Uf and stresses Rf."""
    import torch
    mi, si, mo, so = norm
    Ucl = float(np.max(Uf))
    les = {}
    for name, model in models:
        f = ChannelFlow(gl, re=re, dt=0.005, fix_mass=1, dt_flag=1, cfl_max=cfl, precision=MIXED, device=device)
        f.upload_state(state, None, None)
        sc = f.scalars()
        f.set_scalars(0.0, sc["dt"], sc["p_grad"], wall_gradient(state, gl))
        f.remove_initial_divergence()
        f.compute_initial_pressure(0)
        if model:
            f.set_les(model, cs=cs, beta=beta, mlp=net if model == 2 else None, in_shift=mi, in_scale=si,
                      out_shift=mo, out_scale=so)
        st, e0, e1 = _events(torch, f)
        e0.record(st)
        n1 = advance_to(f, les_spin)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / max(n1, 1)
        ms_tu = e0.elapsed_time(e1) / f.scalars()["t_total"]
        U, R, k, n2 = 0.0, 0.0, 0, 0
        t_end = les_spin + les_avg
        while f.scalars()["t_total"] < t_end - 1e-12 and f.status() == 0:
            n2 += advance_to(f, min(t_end, f.scalars()["t_total"] + 0.5))
            u_, r_ = profile_stats(f.download_state()[0], gl)
            U, R, k = U + u_, R + r_, k + 1
        stt = f.status()
        res = {"status": stt, "ms_per_step": ms, "ms_per_time_unit": ms_tu, "steps_spinup": n1,
               "dt": f.scalars()["dt"]}
        if k and stt == 0:
            U, R = U / k, R / k
            res["mean_profile_max_rel_err"] = float(np.max(np.abs(U - Uf)) / Ucl)
            res["mean_profile_rel_l2"] = float(np.linalg.norm(U - Uf) / np.linalg.norm(Uf))
            res["uv_rel_l2"] = float(np.linalg.norm(R[3] - Rf[3]) / np.linalg.norm(Rf[3]))
            res["uu_rel_l2"] = float(np.linalg.norm(R[0] - Rf[0]) / np.linalg.norm(Rf[0]))
        if model == 2:
            nf, npts = f.les_fallbacks()
            res["fallback_fraction"] = nf / max(1, npts * 3 * (n1 + n2))
        les[name] = res
        log(f"LES {name}: {res}")
        f.close()
    return les


def les_from_artifact(path, device=0, log=print, **kw):
    """les_runs from an artifact run_c4 saved: the filtered initial state,
    the filtered DNS statistics, the trained network and its normalisation."""
    a = np.load(path)
    nx, ny, nz = (int(v) for v in a["grid"])
    gl = Grid(nx, ny, nz, lx=4 * np.pi, lz=2 * np.pi, stretch=float(a["stretch"]))
    net = Mlp(device, a["params"])
    try:
        les = les_runs(gl, float(a["re"]), np.asfortranarray(a["state"].astype(np.complex128)), a["Uf"], a["Rf"], net,
                       (a["mi"], a["si"], a["mo"], a["so"]),
                       device=device, log=log, **kw)
    finally:
        net.close()
    dms = float(a["dns_ms_per_time_unit"])
    return les, {k: dms / v["ms_per_time_unit"] for k, v in les.items()}
