"""COLA time integration (py/fs/cola.py): kick and drift with the 2LPT
trajectory subtracted."""
from . import _fs as c


def kick(particles, a_vel):
    """Updates particle velocities to scale factor a_vel, using the force at
    particles' a_x."""
    c._cola_kick(particles._particles, a_vel)


def drift(particles, a_pos):
    """Updates particle positions to scale factor a_pos."""
    c._cola_drift(particles._particles, a_pos)


def step(particles, a_vel, a_pos):
    """One step of the reference's time loop (script/cola.py:37-44) in one
    call: PM force at a_x, kick to a_vel, drift to a_pos.  The result equals
    fs.pm.force + kick + drift."""
    c._cola_step(particles._particles, a_vel, a_pos)


def velocity(particles):
    """The physical (2LPT-restored) velocity v + Dv dx1 + D2v dx2 at a_x as
    an (np, 3) array (cola_velocity of the reference)."""
    return c._cola_velocity(particles._particles)
