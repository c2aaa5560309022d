"""Helpers to compare unrounded values with numbers the reference printed."""
import math


def half_ulp(printed, sig):
    """Half a unit in the last printed digit of a Fortran E-format number with ``sig`` digits."""
    if printed == 0.0:
        return 0.0
    e = math.floor(math.log10(abs(printed))) + 1
    return 0.5 * 10.0 ** (e - sig)


def agrees(value, printed, sig, abs_floor=0.0, slack=1.0e-3):
    """True when ``value`` rounds to ``printed`` at ``sig`` significant digits (with a tiny slack
    for the binary/decimal boundary) or lies within ``abs_floor`` of it."""
    tol = half_ulp(printed, sig) * (1.0 + slack) + abs(printed) * 1e-12
    return abs(value - printed) <= max(tol, abs_floor)
