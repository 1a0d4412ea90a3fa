"""Attenuation and dispersion of the viscoacoustic scheme, measured by spectral ratios, against the
standard-linear-solid (1 SLS) law with the reference's Blanch tau parameters.

Reference: forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90
  * pcalpas (QS:473-551): Q is scaled by 18/20; tau_sigma = 1 / ((w_up - w_low) / 2) with
    w_low = 2 * 2 pi and w_up = 2.5 f0 * 2 pi; tau = (1/Q') (ln(ts^2 w_up^2 + 1) - ln(ts^2 w_low^2 + 1))
    / (d_up - d_low), d = atan(w ts) - w ts / (1 + ts^2 w^2); tau_eps = tau_sigma (1 + tau);
  * calpstr* / calpr* (QS:993-1269) in the order of extrapolation_one_step (QS:751-835): the stress
    takes sigma += dt (M tau_eps/tau_sigma D + r) with the memory variable of the previous step,
    then r += dt (-1/tau_sigma) (M (tau_eps/tau_sigma - 1) D + r).

Continuous 1-SLS law (e^{i w t}): M(w) = M_R (1 + i w tau_eps) / (1 + i w tau_sigma), with M_R = rho vp^2
the relaxed modulus; Q^-1(w) = Im M / Re M.  The same update in discrete time (z = e^{i w dt},
D at half steps) gives the effective modulus
    M_d(w) = M_R [tau_eps/tau_sigma - (dt/tau_sigma)(tau_eps/tau_sigma - 1) / (z - 1 + dt/tau_sigma)],
which tends to M(w) as dt -> 0 (the explicit memory step is first order in dt/tau_sigma).

Measurement: a homogeneous model, a source and two receivers on one row at offsets r1 < r2.  The
spectral ratio U(r2)/U(r1) of a run with quality factor Q, divided by the same ratio of a run with
Q = 1e5 (no attenuation), cancels the source spectrum, the Gaussian source spread and most of
the grid dispersion.  In 2-D the point-source pressure is H0(k r) (Hankel function; H0^(2) for
e^{i w t}), so the expected ratio of ratios is
    [H0(k_Q r2) / H0(k_Q r1)] / [H0(k_0 r2) / H0(k_0 r1)],   k_Q = (w / vp) sqrt(M_R / M(w)),
near field included.  Its log-amplitude per metre is the attenuation coefficient alpha(w) and
its unwrapped phase per metre the dispersion (the change of Re k); the measured and expected
values are compared over 0.5 f0 .. 2 f0.
"""
import numpy as np
from scipy.special import hankel2

PI_REF = 3.1415926  # the constant module's pi (QS:4)


def blanch_tau(q: float, f0: float):
    """(tau_sigma, tau) of QS:511-542 in double precision (the reference's Q * 18/20 included)."""
    flow = 2 * 2 * PI_REF
    fup = 2.5 * f0 * 2 * PI_REF
    qe = q * (18.0 / 20.0)
    ts = 1.0 / ((fup - flow) / 2.0)
    nlow = np.log(ts ** 2 * flow ** 2 + 1)
    nup = np.log(ts ** 2 * fup ** 2 + 1)
    dlow = np.arctan(flow * ts) - flow * ts / (1 + ts ** 2 * flow ** 2)
    dup = np.arctan(fup * ts) - fup * ts / (1 + ts ** 2 * fup ** 2)
    return ts, (1.0 / qe) * (nup - nlow) / (dup - dlow)


def modulus(w, q, f0, dt=None):
    """M(w) / M_R: the continuous 1-SLS law (dt None) or the discrete-time law of the scheme."""
    ts, tau = blanch_tau(q, f0)
    te_ts = 1.0 + tau
    if dt is None:
        return (1 + 1j * w * ts * te_ts) / (1 + 1j * w * ts)
    z = np.exp(1j * w * dt)
    return te_ts - (dt / ts) * (te_ts - 1) / (z - 1 + dt / ts)


def inverse_q(w, q, f0, dt=None):
    m = modulus(w, q, f0, dt)
    return np.imag(m) / np.real(m)


def _spectrum(trace, dt, t_end, n_fft=8192, taper_s=0.05):
    """Spectrum of a trace cut off at t_end with a cosine taper of taper_s seconds before it."""
    nt = trace.shape[0]
    w = np.ones(nt)
    i1 = min(int(round(t_end / dt)), nt)
    nta = int(round(taper_s / dt))
    w[i1:] = 0.0
    w[max(0, i1 - nta):i1] = 0.5 * (1 + np.cos(np.pi * np.arange(min(nta, i1)) / nta))
    return np.fft.rfft(np.asarray(trace, np.float64) * w, n_fft), np.fft.rfftfreq(n_fft, dt)


def measure(rec_q, rec_0, i1, i2, r1_m, r2_m, vp, f0, dt, q):
    """rec_q / rec_0: records [trace][time] of the Q run and of the Q = 1e5 run (time 0 at the
    wavelet peak); i1 / i2: the traces at offsets r1_m < r2_m (metres) from the source.  Returns a
    dict of per-frequency arrays over 0.5 f0 .. 2 f0: f, measured and expected (continuous and
    discrete law) attenuation coefficients and dispersion, and Q^-1 of both laws."""
    t1 = r1_m / vp + 0.25
    t2 = r2_m / vp + 0.20

    def ratio(rec):
        a, f = _spectrum(rec[i1], dt, t1)
        b, _ = _spectrum(rec[i2], dt, t2)
        return b / a, f

    rq, f = ratio(rec_q)
    r0, _ = ratio(rec_0)
    band = (f >= 0.5 * f0) & (f <= 2.0 * f0)
    w = 2 * np.pi * f[band]
    rr = (rq / r0)[band]
    dr = r2_m - r1_m
    out = {"f": f[band], "alpha": -np.log(np.abs(rr)) / dr, "disp": np.unwrap(np.angle(rr)) / dr}
    k0 = w / vp
    for name, step in (("cont", None), ("disc", dt)):
        kq = k0 / np.sqrt(modulus(w, q, f0, step))
        ana = (hankel2(0, kq * r2_m) / hankel2(0, kq * r1_m)) / (hankel2(0, k0 * r2_m) / hankel2(0, k0 * r1_m))
        out["alpha_" + name] = -np.log(np.abs(ana)) / dr
        out["disp_" + name] = np.unwrap(np.angle(ana)) / dr
        out["qinv_" + name] = inverse_q(w, q, f0, step)
    return out


def rel_err(meas, exp):
    return float(np.max(np.abs(meas / exp - 1.0)))


# The test geometry (interior cells): a homogeneous 260 x 200 model, 30 sponge cells per side, the
# source at interior (x = 60, mid depth), receivers on its row at offsets 30 and 150 cells.  With
# vp = 2000 m/s, dx = 5 m the reflections from the sponges reach the far receiver after 0.62 s,
# later than the analysis windows.
GEOM = dict(nx=260, nz=200, npx=30, sx=60, r1=30, r2=150, dx=5.0, vp=2000.0, rho=2000.0, f0=20.0)
