"""Algorithmic work of the photon march, for roofline figures.

The unit of work is one ER step: the kick-drift-kick leapfrog of renderer/src/scene.cpp:323-330
plus the traceTillBlock bookkeeping of scene.cpp:395-419, with ONE fused evaluation of n and
grad n at the new point (the evaluations at the old point are the previous step's). FLOPs are
counted from the reference's formulas (scene.cpp:206-257 for the Bessel mode), one FLOP per
add/sub/mul/div/sqrt and one per transcendental call (jn, atan2, sin, cos):

  leapfrog             2 kicks x (1 + 3 mul + 3 add) + drift (3 mul + 1 div + 3 mul + 3 add)  = 24
  bookkeeping          6 box subtractions + 1 distance add + distance+=h + total+=h*n (2)       = 10
  Bessel n, grad n     r^2 (3) + sqrt + kr + J_m + J_m+1 (2) + A = n_max*s (1) + n (3)          = 11
                       1/r, 1/r^2 (2); m = 0: grad (2 x 4)                                      = 10
                       m >= 1: atan2, m*phi, cos, sin (4) + J' (3) + grad (2 x 11)              = 31
  mode 0: 55 FLOP/step, mode >= 1: 78 FLOP/step.

  plane waves (each)   phase k.p - tau + phase (7) + sin, cos (2) + n (2) + grad (7)           = 18
                       n = n_o + sum (1): two waves 37, 71 FLOP/step
  tricubic spline      per axis: floor, fraction, 4 weights, 4 derivative weights (25)          = 75
                       16 rows of 4 taps: value and x-derivative sums (14) + y/z/value/x
                       accumulation (11) (spline.h:415-448, separable)                          = 400
                       scale of the gradient (3) + base (1)                                      = 4
                       479, 513 FLOP/step

The adjoint's backward sweep visits every recorded point once (adjoint.cuh): n, grad n and the
Hessian there, the parameter vector-Jacobian product, and the step's own adjoint algebra
(dh, d_prev, Dh, a, b, P += a g + H b for both kicks, about 80 FLOP):
  plane waves (each)   phase (7) + sin, cos (2) + n (2) + grad (7) + Hessian (13)                 = 31
                       parameter product: phase (7) + sin, cos (2) + k.b (5) + two sums (7)      = 21
  tricubic spline      weights of three orders on three axes (72), 16 rows x (three 4-tap sums
                       (21) + ten accumulations (20) + products (3)) (704), scaling (15)        = 791
                       parameter product: weights (72) + 16 rows x (row factors (10) + 4 taps
                       (12)) (352)                                                              = 424
  Bessel m <= 2        r, 1/r (3) + J_m, J_m+1 (2) + cos, sin of m phi (4) + J', J'' (9) + f and
                       the polar derivatives (9) + grad f (8) + Hessian in y, z (21) + scaling
                       by A (8)                                                                  = 64
                       parameter product a f + b . grad f (6)                                    = 6
"""

FLOP_LEAPFROG = 24
FLOP_BOOKKEEPING = 10


def flop_per_step_bessel(mode: int) -> int:
    field = 11 + 2 + (8 if mode == 0 else 31)
    return FLOP_LEAPFROG + FLOP_BOOKKEEPING + field


def flop_per_step_planewave(n_waves: int) -> int:
    return FLOP_LEAPFROG + FLOP_BOOKKEEPING + 18 * n_waves + 1


def flop_per_step_spline() -> int:
    return FLOP_LEAPFROG + FLOP_BOOKKEEPING + 75 + 400 + 4


def flop_per_step_sources(n_coeff: int, n_sources: int, arcs: int) -> int:
    """Point sources (scene.cpp:139-195): per source and harmonic, offset (3), squared distance
    (5), 1/r and r (2), k r c (2), phase + sin, cos (3), value sum (2), radial factor (5),
    gradient sums (6) = 28; per harmonic its weight and the two sums (10); n and the scaled
    gradient (5)."""
    return FLOP_LEAPFROG + FLOP_BOOKKEEPING + n_coeff * (28 * arcs * n_sources + 10) + 5


def flop_per_step(setup) -> int:
    """FLOP per ER step of a Setup's field."""
    from . import _lib as L
    if setup.field_type == L.FIELD_SOURCES:
        arcs = int(bool(setup.active1)) + int(bool(setup.active2))
        return flop_per_step_sources(setup.n_coeff, setup.theta_sources * setup.trans_z_sources, arcs)
    if setup.field_type == L.FIELD_PLANEWAVE:
        return flop_per_step_planewave(len(setup.wave_amp))
    if setup.field_type == L.FIELD_SPLINE:
        return flop_per_step_spline()
    return flop_per_step_bessel(setup.mode)


FLOP_ADJ_STEP = 80


def flop_per_point_adjoint(setup) -> int:
    """FLOP per point of the adjoint's backward sweep."""
    from . import _lib as L
    if setup.field_type == L.FIELD_PLANEWAVE:
        return FLOP_ADJ_STEP + (31 + 21) * len(setup.wave_amp)
    if setup.field_type == L.FIELD_SPLINE:
        return FLOP_ADJ_STEP + 791 + 424
    if setup.field_type == L.FIELD_BESSEL:
        return FLOP_ADJ_STEP + 64 + 6
    raise ValueError("the adjoint is built for Bessel, plane-wave and spline fields")
