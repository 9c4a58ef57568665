"""Analytic response of a homogeneous half-space to a central loop.

Ward & Hohmann (1988), "Electromagnetic theory for geophysical applications",
eq. 4.98: for a horizontal circular loop of radius a carrying a step-off
current I on the surface of a half-space of conductivity sigma, the time
derivative of the vertical magnetic field at the loop centre is

    dh_z/dt = -I / (sigma mu0 a^3) [3 erf(theta a)
              - 2/sqrt(pi) theta a (3 + 2 theta^2 a^2) exp(-theta^2 a^2)],
    theta = sqrt(mu0 sigma / (4 t)),

so dB_z/dt = mu0 dh_z/dt.  A step-on source gives the negated response once
the turn-on ramp is over (linearity).  Used only by the tests.
"""
import math

import numpy as np

MU0 = 4e-7 * math.pi


def central_loop_dbzdt(t, sigma: float, radius: float, current: float = 1.0):
    """dB_z/dt (T/s) at the centre of a step-off loop on a half-space."""
    t = np.asarray(t, dtype=np.float64)
    from scipy.special import erf
    ta = np.sqrt(MU0 * sigma / (4.0 * t)) * radius
    br = 3.0 * erf(ta) - 2.0 / math.sqrt(math.pi) * ta * (3.0 + 2.0 * ta * ta) * np.exp(-ta * ta)
    return -current / (sigma * radius ** 3) * br


def erf_step_on_dbzdt(t, sigma: float, radius: float, t0: float, current: float = 1.0, n: int = 64):
    """dB_z/dt for the reference's erf step-on waveform (pulse type 1, whose
    dI/dt is 5/(sqrt(pi) t0) exp(-25 (tau - t0/2)^2 / t0^2) I, a Gaussian
    over [0, t0]): the step-off response convolved with dI/dt and negated,
    by Gauss-Legendre quadrature over [0, t0].  Valid for t > t0."""
    t = np.atleast_1d(np.asarray(t, dtype=np.float64))
    xg, wg = np.polynomial.legendre.leggauss(n)
    tau = 0.5 * t0 * (xg + 1.0)
    w = 0.5 * t0 * wg * 5.0 / (math.sqrt(math.pi) * t0) * np.exp(-25.0 * (tau - 0.5 * t0) ** 2 / (t0 * t0))
    out = np.zeros_like(t)
    for i, ti in enumerate(t):
        out[i] = -np.sum(w * central_loop_dbzdt(ti - tau, sigma, radius, current))
    return out
