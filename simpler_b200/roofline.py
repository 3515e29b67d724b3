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
"""

FLOP_LEAPFROG = 24
FLOP_BOOKKEEPING = 10


def flop_per_step_bessel(mode: int) -> int:
    field = 11 + 2 + (8 if mode == 0 else 31)
    return FLOP_LEAPFROG + FLOP_BOOKKEEPING + field
