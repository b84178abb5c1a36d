"""Linear P(k) tables for the synthetic inputs: the Eisenstein & Hu (1998,
ApJ 496, 605) "no-wiggle" transfer function, eqs. 26-31, normalised to a
given sigma_8 with the same trapezoid sum the reference uses
(PowerSpectrum::compute_sigma, py/power.cpp:146-170), and written as the
two-column `k P` text table that PowerSpectrum::read_file_ reads
(py/power.cpp:57-144; k in h/Mpc, P in (Mpc/h)^3, linear at a=1).
"""
from __future__ import annotations

import math

import numpy as np

T_CMB = 2.7255


def transfer_nowiggle(k_h: np.ndarray, omega_m: float, omega_b: float,
                      h: float) -> np.ndarray:
    """EH98 zero-baryon-oscillation transfer function T0(k); k in h/Mpc."""
    theta = T_CMB / 2.7
    om_h2 = omega_m * h * h
    ob_h2 = omega_b * h * h
    fb = omega_b / omega_m
    # sound horizon fit, eq. 26 [Mpc]
    s = 44.5 * math.log(9.83 / om_h2) / math.sqrt(1.0 + 10.0 * ob_h2 ** 0.75)
    # eq. 31
    alpha = (1.0 - 0.328 * math.log(431.0 * om_h2) * fb
             + 0.38 * math.log(22.3 * om_h2) * fb * fb)
    k_mpc = k_h * h
    gamma_eff = omega_m * h * (alpha + (1.0 - alpha) /
                               (1.0 + (0.43 * k_mpc * s) ** 4))   # eq. 30
    q = k_h * theta * theta / gamma_eff                           # eq. 28
    L0 = np.log(2.0 * math.e + 1.8 * q)                           # eq. 29
    C0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return L0 / (L0 + C0 * q * q)


def sigma_trapezoid(k: np.ndarray, P: np.ndarray, R: float) -> float:
    """sigma_R by the trapezoid rule over the table, as
    PowerSpectrum::compute_sigma does (first step from k[0] with f0 = 0)."""
    x = k * R
    w = 3.0 * (np.sin(x) - x * np.cos(x)) / (x * x * x)
    f = P * k * k * w * w
    f_prev = np.concatenate([[0.0], f[:-1]])
    k_prev = np.concatenate([[k[0]], k[:-1]])
    s2 = np.sum(0.5 * (f_prev + f) * (k - k_prev))
    return math.sqrt(s2 / (2.0 * math.pi * math.pi))


def eh_nowiggle_table(omega_m: float = 0.31, omega_b: float = 0.049,
                      h: float = 0.67, n_s: float = 0.96,
                      sigma8: float = 0.81, k_min: float = 1e-4,
                      k_max: float = 1e3, n: int = 1000):
    """(k, P) arrays, log-spaced in k, normalised to sigma8."""
    k = np.logspace(math.log10(k_min), math.log10(k_max), n)
    T = transfer_nowiggle(k, omega_m, omega_b, h)
    P = k ** n_s * T * T
    P *= (sigma8 / sigma_trapezoid(k, P, 8.0)) ** 2
    return k, P


def write_table(filename: str, k: np.ndarray, P: np.ndarray,
                header: str | None = None) -> str:
    with open(filename, "w") as fp:
        if header:
            for line in header.splitlines():
                fp.write("# %s\n" % line)
        for ki, Pi in zip(k, P):
            fp.write("%.10e %.10e\n" % (ki, Pi))
    return filename


def write_eh_nowiggle(filename: str, **kw) -> str:
    k, P = eh_nowiggle_table(**kw)
    params = dict(omega_m=0.31, omega_b=0.049, h=0.67, n_s=0.96, sigma8=0.81)
    params.update({a: b for a, b in kw.items() if a in params})
    hdr = ("Eisenstein-Hu no-wiggle linear P(k) at a=1: "
           + " ".join("%s=%g" % kv for kv in params.items())
           + "\ncolumns: k [h/Mpc]  P [(Mpc/h)^3]")
    return write_table(filename, k, P, hdr)
