"""2LPT initial conditions (py/fs/lpt.py)."""
import numpy as np

from . import _fs as c
from .particles import Particles


def init(nc, boxsize, a, ps, seed, kind):
    """Generates a Gaussian random field and a grid of nc^3 particles with
    2LPT displacements at scale factor a.

    Args:
        nc (int): particles per dimension.
        boxsize (float): periodic box length [Mpc/h].
        a (float): scale factor of the positions.
        ps (PowerSpectrum): linear P(k) at a = 1.
        seed (int): random seed of the field.
        kind (str): 'zeldovich', '2lpt' or 'cola' (cola sets v = 0).

    The field's uniform draws come from this library's counter-based
    generator, not from GSL's ranlxd1, so a seed gives a different (equally
    distributed) realisation than the reference's.  draws(nc, seed) returns
    them; init_from_draws() takes any.

    Returns:
        Particles.
    """
    return Particles(_particles=c._lpt(nc, boxsize, a, seed, ps._ps,
                                       kind.lower()))


def init_from_draws(nc, boxsize, a, ps, u_phase, u_ampl, kind):
    """init() with the uniform draws of every mode given: u_phase and u_ampl
    are (nc, nc, nc//2) arrays in (0, 1], the (phase, amplitude) draws of
    column (ix, iy) at iz."""
    return Particles(_particles=c._lpt_from_draws(
        nc, boxsize, a, np.ascontiguousarray(u_phase, dtype=np.float64),
        np.ascontiguousarray(u_ampl, dtype=np.float64), ps._ps, kind.lower()))


def init_from_delta_k(nc, boxsize, a, delta_k, kind):
    """init() from an unnormalised density field delta(k), an (nc, nc,
    nc//2+1) complex64 half spectrum (e.g. of white noise scaled by
    sqrt(P/V))."""
    return Particles(_particles=c._lpt_from_delta_k(
        nc, boxsize, a, np.ascontiguousarray(delta_k, dtype=np.complex64),
        kind.lower()))


def draws(nc, seed):
    """(u_phase, u_ampl) that init(nc, ..., seed, ...) uses."""
    return c._lpt_draws(nc, seed)


def set_offset(offset):
    """Sets the offset of the particle grid, x = (ix + offset)*boxsize/nc."""
    c._lpt_set_offset(offset)


def set_zeldovich_force(particles, a):
    """Sets particles.force to the Zel'dovich force D(a) dx1."""
    c._lpt_set_zeldovich_force(particles._particles, a)
