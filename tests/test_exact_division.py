"""Proof, by exhaustion with exact rational arithmetic, that the kernel's
FMA-corrected quotient (q = x*r, e = fma(-q, d, x), q' = fma(e, r, q), with r
the float nearest 1/d) equals the correctly rounded x / d on every value the
v11 features can divide: holes (<= 230) / 20, hole depths (<= 2599) / 200,
wells (<= 10) / 5 and sqrt(surface sum <= 4761) / 100. The IEEE fma rounds once,
so each step is modelled as one rounding of the exact rational result."""
from __future__ import annotations

from fractions import Fraction as F

import numpy as np

f32 = np.float32


def rn32(fr: F) -> np.float32:
    c = f32(float(fr))
    best = None
    for cand in (np.nextafter(c, f32(-np.inf)), c, np.nextafter(c, f32(np.inf))):
        d = abs(F(float(cand)) - fr)
        if best is None or d < best[0] or (d == best[0] and (int(cand.view(np.uint32)) & 1) == 0):
            best = (d, cand)
    return best[1]


def corrected_quotient_exact(xs, d) -> bool:
    r = rn32(F(1, d))
    R = F(float(r))
    for x in xs:
        X = F(float(f32(x)))
        q = rn32(X * R)
        e = rn32(X - F(float(q)) * d)
        q2 = rn32(F(float(e)) * R + F(float(q)))
        if q2.view(np.uint32) != rn32(X / d).view(np.uint32):
            return False
    return True


def test_reciprocals_are_the_kernel_constants():
    assert rn32(F(1, 20)) == f32(0.05) and rn32(F(1, 200)) == f32(0.005)
    assert rn32(F(1, 5)) == f32(0.2) and rn32(F(1, 100)) == f32(0.01)


def test_holes_wells_hole_depths():
    assert corrected_quotient_exact(range(0, 231), 20)
    assert corrected_quotient_exact(range(0, 11), 5)
    assert corrected_quotient_exact(range(0, 2600), 200)


def test_surface_sqrt():
    # sqrt(s) for integer s < 2^24 rounded once: take the float32 nearest the true root
    roots = []
    for s in range(0, 4762):
        c = f32(np.sqrt(np.float64(s)))
        best = min((np.nextafter(c, f32(-1)), c, np.nextafter(c, f32(1e9))),
                   key=lambda t: abs(F(float(t)) ** 2 - s) if s else abs(F(float(t))))
        roots.append(best)
    assert corrected_quotient_exact(roots, 100)
