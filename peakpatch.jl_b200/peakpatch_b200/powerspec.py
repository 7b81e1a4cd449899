"""Tabulated linear power spectra for run_tile's `pkfile`.

The reference reads P(k) from a two-column file (k in h/Mpc, P) and
interpolates it log-log (src/InitialConditions/PowerSpectrum.jl:11-30).  It
contains no power-spectrum model of its own; this module writes such files
from the Eisenstein & Hu (1998, ApJ 496, 605) "no-wiggle" transfer function,
eqs. (26)-(31), with a primordial tilt n_s and a sigma_8 normalisation.

File convention.  The reference scales white noise by sqrt(P(k) dk^3 n^3)
(RandomField.jl:165), so the real-space variance of the field is
sum_k P(k) dk^3 ~ integral P d^3k.  For a spectrum P_std normalised the usual
way, sigma^2 = integral P_std d^3k / (2 pi)^3, the file therefore holds
P_std / (2 pi)^3.
"""
from __future__ import annotations

import numpy as np

T_CMB = 2.7255


def eh_nowiggle_transfer(k_hmpc: np.ndarray, Om: float, Ob: float, h: float) -> np.ndarray:
    """Eisenstein & Hu (1998) zero-baryon-shape transfer function with the
    baryon suppression of the effective shape (eqs. 26, 28-31)."""
    k = np.asarray(k_hmpc, dtype=np.float64)
    theta = T_CMB / 2.7
    om_h2 = Om * h * h
    ob_h2 = Ob * h * h
    fb = Ob / Om
    s = 44.5 * np.log(9.83 / om_h2) / np.sqrt(1.0 + 10.0 * ob_h2 ** 0.75)           # Mpc, eq. 26
    alpha = 1.0 - 0.328 * np.log(431.0 * om_h2) * fb + 0.38 * np.log(22.3 * om_h2) * fb * fb   # eq. 31
    k_mpc = k * h
    gamma = Om * h * (alpha + (1.0 - alpha) / (1.0 + (0.43 * k_mpc * s) ** 4))        # eq. 30
    q = k * theta * theta / gamma                                                        # eq. 28
    L0 = np.log(2.0 * np.e + 1.8 * q)
    C0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return L0 / (L0 + C0 * q * q)                                                        # eq. 29


def tophat_w(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    m = x > 1e-6
    xm = x[m]
    out[m] = 3.0 * (np.sin(xm) - xm * np.cos(xm)) / xm ** 3
    return out


def sigma_R(k: np.ndarray, P_std: np.ndarray, R: float) -> float:
    """sigma(R) of a spectrum tabulated on a log grid (standard convention)."""
    lk = np.log(k)
    integrand = k ** 3 * P_std * tophat_w(k * R) ** 2 / (2.0 * np.pi ** 2)
    return float(np.sqrt(np.trapezoid(integrand, lk)))


def eh_table(Om: float = 0.315, Ob: float = 0.049, h: float = 0.674, ns: float = 0.965, sigma8: float = 0.808,
             kmin: float = 1e-5, kmax: float = 1e2, nk: int = 500):
    """(k, P_file) on nk log-spaced points; P_file = P_std / (2 pi)^3 with
    P_std normalised to sigma8 (top-hat, R = 8 Mpc/h)."""
    k = np.logspace(np.log10(kmin), np.log10(kmax), nk)
    # normalise on a finer grid than the table for an accurate integral
    kf = np.logspace(-6, 3, 20000)
    Pf = kf ** ns * eh_nowiggle_transfer(kf, Om, Ob, h) ** 2
    amp = (sigma8 / sigma_R(kf, Pf, 8.0)) ** 2
    P_std = amp * k ** ns * eh_nowiggle_transfer(k, Om, Ob, h) ** 2
    return k, P_std / (2.0 * np.pi) ** 3


def write_pk(path: str, k: np.ndarray, P: np.ndarray, header: str = "") -> None:
    with open(path, "w") as f:
        if header:
            for line in header.splitlines():
                f.write(f"# {line}\n")
        for kk, pp in zip(k, P):
            f.write(f"{float(kk)!r}  {float(pp)!r}\n")


def rescale_sigma8(P: np.ndarray, sigma8_new: float, sigma8_ref: float = 0.808) -> np.ndarray:
    """The serving workload varies sigma8 by rescaling the table."""
    return P * (sigma8_new / sigma8_ref) ** 2
