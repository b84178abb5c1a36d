"""Flat LCDM growth factors (py/fs/cosmology.py), computed on the host in
double precision by libfs2gpu."""
from . import _fs as c


def init(omega_m):
    """Initialises the cosmology module with Omega_m at a = 1."""
    c._cosmology_init(omega_m)


def D_growth(a):
    """Linear growth factor D(a), normalised to D(1) = 1."""
    return c._cosmology_D_growth(a)


def D2_growth(a):
    """Second-order growth factor D2(a); the 2LPT displacement is
    D*dx1 + D2*dx2."""
    return c._cosmology_D2_growth(a)
