"""Mie series of a homogeneous sphere: efficiencies and forward / backward amplitudes.

The sweep driver writes, next to every DDA result, the Mie values of the
volume-equivalent sphere, as the reference's sweep does (run_dda.py:118-123
calling analytical_scattering_theories/homogeneous_sphere.py:4-117).  This is
host arithmetic outside the solve; it follows the published series of
Bohren & Huffman, *Absorption and Scattering of Light by Small Particles*
(1983), section 4.4 and appendix A:

* partial waves n = 1 .. n_stop, n_stop = floor(x + 4 x^(1/3) + 2);
* logarithmic derivative D_n(m x) by downward recurrence
  D_{n-1} = n/(mx) - 1/(D_n + n/(mx)) from n_max = max(n_stop, |mx|) + 15;
* Riccati-Bessel psi_n, chi_n by upward recurrence (stable for n <= n_stop);
* a_n, b_n from eq. 4.88; Q_ext, Q_sca from eqs. 4.61-4.62;
* the amplitudes only at theta = 0 and pi, where pi_n and tau_n are closed
  forms (both n(n+1)/2 at theta = 0; (-1)^(n+1) n(n+1)/2 and (-1)^n n(n+1)/2
  at theta = pi), so no angular recurrence is needed.

Conventions as the reference: medium non-absorbing, S11 = S2 / (-i k),
S22 = S1 / (-i k) with k the wavenumber in the medium; PCAS forward
observable S_fw = (S11(0) + S22(0)) / 2, OCBS backward observable
S_bk = (-S11(pi) + S22(pi)) / sqrt(2).  The reference rounds S_fw and S_bk to
complex64; these are returned in complex128.
"""
from __future__ import annotations

import numpy as np


def mie_q_and_s(wl_0: float, m_m: float, r_p: float, m_p: complex):
    """(Q_sca, Q_abs, Q_ext, S_fw, S_bk) of a sphere of radius r_p and index m_p in a medium m_m."""
    k = 2.0 * np.pi * m_m / wl_0
    x = k * r_p
    m = complex(m_p) / m_m
    mx = m * x
    n_stop = int(np.floor(x + 4.0 * x ** (1.0 / 3.0) + 2.0))
    n_max = int(np.floor(max(n_stop, abs(mx)) + 15))
    D = np.zeros(n_max + 1, dtype=np.complex128)
    for n in range(n_max, 0, -1):
        D[n - 1] = n / mx - 1.0 / (D[n] + n / mx)
    psi = np.empty(n_stop + 1)
    chi = np.empty(n_stop + 1)
    psi[0], chi[0] = np.sin(x), np.cos(x)          # psi_0 = sin x, chi_0 = cos x (BH83 appendix A)
    psi_m1, chi_m1 = np.cos(x), -np.sin(x)         # n = -1
    for n in range(1, n_stop + 1):
        prev_p = psi[n - 2] if n >= 2 else psi_m1
        prev_c = chi[n - 2] if n >= 2 else chi_m1
        psi[n] = (2 * n - 1) / x * psi[n - 1] - prev_p
        chi[n] = (2 * n - 1) / x * chi[n - 1] - prev_c
    n = np.arange(1, n_stop + 1, dtype=np.float64)
    xi = psi - 1j * chi                            # xi_n = psi_n - i chi_n (BH83 chi sign convention)
    Dn = D[1:n_stop + 1]
    an = ((Dn / m + n / x) * psi[1:] - psi[:-1]) / ((Dn / m + n / x) * xi[1:] - xi[:-1])
    bn = ((m * Dn + n / x) * psi[1:] - psi[:-1]) / ((m * Dn + n / x) * xi[1:] - xi[:-1])
    w = 2.0 * n + 1.0
    q_ext = float(2.0 / x ** 2 * np.sum(w * (an + bn).real))
    q_sca = float(2.0 / x ** 2 * np.sum(w * (np.abs(an) ** 2 + np.abs(bn) ** 2)))
    sign = np.where(n % 2 == 1, 1.0, -1.0)         # (-1)^(n+1)
    s1_0 = np.sum(w / 2.0 * (an + bn))             # = S2(0)
    s1_pi = np.sum(w / 2.0 * sign * (an - bn))     # S2(pi) = -S1(pi)
    mik = -1j * k
    s_fw = s1_0 / mik
    s_bk = (s1_pi + s1_pi) / mik / np.sqrt(2.0)    # (-S11(pi) + S22(pi)) / sqrt 2, S11(pi) = -S1(pi)/(-ik)
    return q_sca, q_ext - q_sca, q_ext, complex(s_fw), complex(s_bk)
