"""Exact solution of the 1-D Euler Riemann problem (Toro, "Riemann Solvers and Numerical Methods
for Fluid Dynamics", ch. 4: Newton iteration on the pressure function, then sampling)."""
import numpy as np


def _f(p, rho, P, c, g):
    if p > P:   # shock
        A = 2 / ((g + 1) * rho)
        B = (g - 1) / (g + 1) * P
        q = np.sqrt(A / (p + B))
        return (p - P) * q, q * (1 - (p - P) / (2 * (B + p)))
    r = p / P   # rarefaction
    return 2 * c / (g - 1) * (r ** ((g - 1) / (2 * g)) - 1), 1 / (rho * c) * r ** (-(g + 1) / (2 * g))


def star(rl, ul, pl, rr, ur, pr, g):
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        pn = p - (fl + fr + ur - ul) / (dl + dr)
        pn = max(pn, 1e-12)
        if abs(pn - p) < 1e-14 * p:
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(x, t, x0, rl, ul, pl, rr, ur, pr, g):
    """Density, velocity, pressure at positions x and time t (interface at x0)."""
    ps, us = star(rl, ul, pl, rr, ur, pr, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for i, xi in enumerate(x):
        s = (xi - x0) / t
        if s <= us:   # left of contact
            if ps > pl:   # left shock
                sl = ul - cl * np.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    out[:, i] = (rl, ul, pl)
                else:
                    r = rl * (ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1)
                    out[:, i] = (r, us, ps)
            else:         # left rarefaction
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    out[:, i] = (rl, ul, pl)
                elif s >= stl:
                    out[:, i] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    out[:, i] = (rl * (c / cl) ** (2 / (g - 1)), u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:
            if ps > pr:   # right shock
                sr = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    out[:, i] = (rr, ur, pr)
                else:
                    r = rr * (ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1)
                    out[:, i] = (r, us, ps)
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    out[:, i] = (rr, ur, pr)
                elif s <= str_:
                    out[:, i] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    out[:, i] = (rr * (c / cr) ** (2 / (g - 1)), u, pr * (c / cr) ** (2 * g / (g - 1)))
    return out
