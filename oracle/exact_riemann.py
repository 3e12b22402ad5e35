"""Exact solution of the 1D Euler Riemann problem (Toro, ch. 4) -- TEST INFRASTRUCTURE ONLY.

Restates the reference's experiments/plot_sod.py:12-65 (f_K pressure functions, brentq root for p*,
u* = mean + half the f_K difference, then the wave-fan sampling), without its plotting imports.
Used for the Sod known answers p* = 0.30313, u* = 0.92745, rho*_R = 0.26557 and L1 errors.
"""
import numpy as np
from scipy.optimize import brentq

G = 1.4


def f_K(p, rho, pK, a):
    if p > pK:  # shock
        A = 2.0 / ((G + 1) * rho)
        B = (G - 1) / (G + 1) * pK
        return (p - pK) * np.sqrt(A / (p + B))
    return 2 * a / (G - 1) * ((p / pK) ** ((G - 1) / (2 * G)) - 1)  # rarefaction


def star_state(left, right):
    rhoL, uL, pL = left
    rhoR, uR, pR = right
    aL, aR = np.sqrt(G * pL / rhoL), np.sqrt(G * pR / rhoR)
    ps = brentq(lambda p: f_K(p, rhoL, pL, aL) + f_K(p, rhoR, pR, aR) + (uR - uL), 1e-10, 10 * max(pL, pR))
    us = 0.5 * (uL + uR) + 0.5 * (f_K(ps, rhoR, pR, aR) - f_K(ps, rhoL, pL, aL))
    return ps, us


def exact_riemann(left, right, x, x0, t):
    """Returns ((len(x), 3) array of rho, u, p, p*, u*)."""
    rhoL, uL, pL = left
    rhoR, uR, pR = right
    aL, aR = np.sqrt(G * pL / rhoL), np.sqrt(G * pR / rhoR)
    ps, us = star_state(left, right)
    gm = (G - 1) / (G + 1)
    out = np.zeros((len(x), 3))
    for k, xi in enumerate(x):
        S = (xi - x0) / t
        if S <= us:
            if ps > pL:
                SL = uL - aL * np.sqrt((G + 1) / (2 * G) * ps / pL + (G - 1) / (2 * G))
                out[k] = left if S <= SL else (rhoL * (ps / pL + gm) / (gm * ps / pL + 1), us, ps)
            else:
                SHL, STL = uL - aL, us - aL * (ps / pL) ** ((G - 1) / (2 * G))
                if S <= SHL:
                    out[k] = left
                elif S > STL:
                    out[k] = (rhoL * (ps / pL) ** (1 / G), us, ps)
                else:
                    c = 2 / (G + 1) * (aL + (G - 1) / 2 * (uL - S))
                    out[k] = (rhoL * (c / aL) ** (2 / (G - 1)), 2 / (G + 1) * (aL + (G - 1) / 2 * uL + S),
                              pL * (c / aL) ** (2 * G / (G - 1)))
        else:
            if ps > pR:
                SR = uR + aR * np.sqrt((G + 1) / (2 * G) * ps / pR + (G - 1) / (2 * G))
                out[k] = right if S >= SR else (rhoR * (ps / pR + gm) / (gm * ps / pR + 1), us, ps)
            else:
                SHR, STR = uR + aR, us + aR * (ps / pR) ** ((G - 1) / (2 * G))
                if S >= SHR:
                    out[k] = right
                elif S <= STR:
                    out[k] = (rhoR * (ps / pR) ** (1 / G), us, ps)
                else:
                    c = 2 / (G + 1) * (aR - (G - 1) / 2 * (uR - S))
                    out[k] = (rhoR * (c / aR) ** (2 / (G - 1)), 2 / (G + 1) * (-aR + (G - 1) / 2 * uR + S),
                              pR * (c / aR) ** (2 * G / (G - 1)))
    return out, ps, us
