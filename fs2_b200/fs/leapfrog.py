"""Leapfrog (non-COLA) time integration (py/fs/leapfrog.py): the plain
kick-drift-kick integrator, without the 2LPT trajectory subtracted."""
from . import _fs as c


def initial_velocity(particles, a_vel):
    """Sets the velocities to the 2LPT velocity dx1 Dv + dx2 D2v at a_vel
    (for particles made with kind='cola', whose v starts at 0)."""
    c._leapfrog_initial_velocity(particles._particles, a_vel)


def kick(particles, a_vel):
    """Updates particle velocities to scale factor a_vel, using the force at
    particles' a_x."""
    c._leapfrog_kick(particles._particles, a_vel)


def drift(particles, a_pos):
    """Updates particle positions to scale factor a_pos."""
    c._leapfrog_drift(particles._particles, a_pos)
