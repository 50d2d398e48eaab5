"""Mie-series efficiencies of a homogeneous sphere -- TEST INFRASTRUCTURE ONLY.

A physics reference for the DDA checks (not a parity oracle: the DDA of a
staircase sphere differs from the exact sphere by its discretisation error).
Only ``tests/`` import it.

Algorithm: the series of Bohren & Huffman, "Absorption and Scattering of Light
by Small Particles" (Wiley 1983), chapter 4 and appendix A: the logarithmic
derivative D_n(mx) by downward recurrence from n_mx = max(n_stop, |mx|) + 15
with D = 0, the Riccati-Bessel functions psi_n(x) = x j_n(x) and
chi_n(x) = -x y_n(x) by upward recurrence from psi_{-1} = cos x,
psi_0 = sin x, chi_{-1} = -sin x, chi_0 = cos x, xi_n = psi_n - i chi_n,
n_stop = x + 4 x^(1/3) + 2, and

  a_n = [(D_n/m + n/x) psi_n - psi_{n-1}] / [(D_n/m + n/x) xi_n - xi_{n-1}]
  b_n = [(m D_n + n/x) psi_n - psi_{n-1}] / [(m D_n + n/x) xi_n - xi_{n-1}]
  Q_ext = 2/x^2 sum (2n+1) Re(a_n + b_n)
  Q_sca = 2/x^2 sum (2n+1) (|a_n|^2 + |b_n|^2)
  g Q_sca = 4/x^2 sum [ n(n+2)/(n+1) Re(a_n a*_{n+1} + b_n b*_{n+1})
                        + (2n+1)/(n(n+1)) Re(a_n b*_n) ]
"""
from __future__ import annotations

import math

import numpy as np


def mie_efficiencies(x: float, m: complex):
    """(Q_ext, Q_sca, Q_abs, g) of a sphere of size parameter x = k a and
    relative refractive index m (Im m >= 0)."""
    x = float(x)
    m = complex(m)
    y = m * x
    nstop = int(round(x + 4.0 * x ** (1.0 / 3.0) + 2.0))
    nmx = int(round(max(nstop, abs(y)))) + 15
    d = np.zeros(nmx + 1, dtype=complex)
    for n in range(nmx, 0, -1):
        d[n - 1] = n / y - 1.0 / (d[n] + n / y)
    psi0, psi1 = math.cos(x), math.sin(x)   # psi_{-1}, psi_0
    chi0, chi1 = -math.sin(x), math.cos(x)  # chi_{-1}, chi_0
    xi1 = complex(psi1, -chi1)
    a = np.zeros(nstop + 2, dtype=complex)
    b = np.zeros(nstop + 2, dtype=complex)
    for n in range(1, nstop + 1):
        psi = (2.0 * n - 1.0) / x * psi1 - psi0
        chi = (2.0 * n - 1.0) / x * chi1 - chi0
        xi = complex(psi, -chi)
        ta = d[n] / m + n / x
        tb = m * d[n] + n / x
        a[n] = (ta * psi - psi1) / (ta * xi - xi1)
        b[n] = (tb * psi - psi1) / (tb * xi - xi1)
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
    n = np.arange(1, nstop + 1)
    an, bn = a[1:nstop + 1], b[1:nstop + 1]
    qext = 2.0 / x ** 2 * float(np.sum((2 * n + 1) * (an + bn).real))
    qsca = 2.0 / x ** 2 * float(np.sum((2 * n + 1) * (np.abs(an) ** 2 + np.abs(bn) ** 2)))
    an1, bn1 = a[2:nstop + 2], b[2:nstop + 2]  # a_{n+1}, b_{n+1} (zero beyond nstop)
    gq = 4.0 / x ** 2 * float(np.sum(n * (n + 2) / (n + 1) * (an * np.conj(an1) + bn * np.conj(bn1)).real
                                     + (2 * n + 1) / (n * (n + 1)) * (an * np.conj(bn)).real))
    return qext, qsca, qext - qsca, gq / qsca


def mie_amplitudes(x: float, m: complex, theta):
    """Amplitude functions S1(theta), S2(theta) of the sphere (Bohren & Huffman
    eq. 4.74) with the angular functions pi_n, tau_n of their eq. 4.47:
    pi_0 = 0, pi_1 = 1, pi_n = (2n-1)/(n-1) mu pi_{n-1} - n/(n-1) pi_{n-2},
    tau_n = n mu pi_n - (n+1) pi_{n-1}, mu = cos(theta)."""
    x = float(x)
    m = complex(m)
    y = m * x
    nstop = int(round(x + 4.0 * x ** (1.0 / 3.0) + 2.0))
    nmx = int(round(max(nstop, abs(y)))) + 15
    d = np.zeros(nmx + 1, dtype=complex)
    for n in range(nmx, 0, -1):
        d[n - 1] = n / y - 1.0 / (d[n] + n / y)
    mu = np.cos(np.asarray(theta, dtype=np.float64))
    s1 = np.zeros(mu.shape, dtype=complex)
    s2 = np.zeros(mu.shape, dtype=complex)
    psi0, psi1 = math.cos(x), math.sin(x)
    chi0, chi1 = -math.sin(x), math.cos(x)
    xi1 = complex(psi1, -chi1)
    pi0, pi1 = np.zeros_like(mu), np.ones_like(mu)  # pi_{n-1}, pi_n for n = 1
    for n in range(1, nstop + 1):
        psi = (2.0 * n - 1.0) / x * psi1 - psi0
        chi = (2.0 * n - 1.0) / x * chi1 - chi0
        xi = complex(psi, -chi)
        ta = d[n] / m + n / x
        tb = m * d[n] + n / x
        an = (ta * psi - psi1) / (ta * xi - xi1)
        bn = (tb * psi - psi1) / (tb * xi - xi1)
        tau = n * mu * pi1 - (n + 1) * pi0
        fn = (2.0 * n + 1.0) / (n * (n + 1.0))
        s1 += fn * (an * pi1 + bn * tau)
        s2 += fn * (an * tau + bn * pi1)
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
        pi0, pi1 = pi1, ((2.0 * n + 1.0) / n) * mu * pi1 - ((n + 1.0) / n) * pi0
    return s1, s2
