"""Particle-mesh force (py/fs/pm.py)."""
from . import _fs as c
from .fft import FFT


def init(nc_pm, pm_factor, boxsize):
    """Initialises the PM module.

    Args:
        nc_pm (int): mesh cells per dimension.
        pm_factor (float): nc_pm / nc, mesh cells per particle spacing.
        boxsize (float): periodic box length.
    """
    c._pm_init(nc_pm, pm_factor, boxsize)


def force(particles):
    """Computes particles.force from particles.x (wrap, CIC density, Poisson
    force on the mesh, CIC interpolation)."""
    send_positions(particles)
    compute_density(particles)
    check_total_density()
    compute_force(particles)
    get_forces(particles)


def send_positions(particles):
    """Wraps positions into the periodic box.  (On one GPU there are no other
    ranks to send boundary particles to.)"""
    c._pm_send_positions(particles._particles)


def compute_density(particles):
    """Computes the CIC density contrast mesh from particles.x; returns it as
    an FFT handle."""
    return FFT(c._pm_compute_density(particles._particles))


def check_total_density():
    """Checks <delta> = 0 when checking is on (set_check(True)); a no-op
    otherwise, as in the reference's default build.

    Raises:
        AssertionError: if the sum is off by more than float precision.
    """
    c._pm_check_total_density()


def compute_force(particles):
    """Computes particles.force from the density mesh."""
    c._pm_compute_force(particles._particles)


def get_forces(particles):
    """Collects forces of particles held by other ranks (none on one GPU)."""
    c._pm_get_forces(particles._particles)


def domain_init(particles):
    """Domain decomposition set-up; nothing to do on one GPU."""
    c._pm_domain_init(particles._particles)


def set_packet_size(packet_size):
    """Halo packet size; nothing to do on one GPU."""
    c._pm_set_packet_size(packet_size)


def set_deposit_mode(mode):
    """'atomic' (default; float atomics) or 'deterministic' (sort by cell and
    fixed-order sums: bitwise reproducible)."""
    c._pm_set_deposit_mode(mode)


def set_bin_tile(shape=-1):
    """Tile (bin) shape of the deterministic deposit: -1 (default) lets the
    autotuner pick at the first deterministic deposit of each mesh and
    particle count; 0..4 fix 16x16x32, 16x8x32, 8x8x32, 8x8x16 or 4x4x32
    cells.  The density is bit for bit the same with every shape."""
    c._pm_set_bin_tile(int(shape))


def bin_tile():
    """(shape, tx, ty, tz) the last deterministic deposit used; shape -1
    before the first."""
    return c._pm_bin_tile()


def set_check(on):
    """Turns the <delta> = 0 check of check_total_density() on or off."""
    c._pm_set_check(bool(on))


def free():
    """Releases the PM mesh and its buffers (pm_free, py/pm.cpp:270)."""
    c._pm_free()


def set_fft_engine(engine):
    """'auto' (default): the faster engine for the mesh, measured on B200:
    the fused five-pass FFT pipeline for 1024^3 meshes, cuFFT otherwise;
    'fused': the fused pipeline for any power-of-two mesh of 64..1024
    cells (cuFFT for other sizes); 'cufft': always cuFFT.  Takes effect at
    the next init() with new arguments."""
    c._pm_set_fft_engine(engine)


def set_fft_tile(columns):
    """Tile width (4 or 8 kz columns) of the fused pipeline's y and x passes;
    a performance parameter only."""
    c._pm_set_fft_tile(columns)


def set_keep_delta_k(on):
    """Keep delta(k) in GPU memory during compute_force so that delta_k()
    can return it (the fused pipeline otherwise never stores it)."""
    c._pm_set_keep_delta_k(bool(on))


def fused():
    """True if the fused FFT pipeline serves the current PM mesh."""
    return c._pm_fused()


def delta_k():
    """The unnormalised density spectrum of the last force computation, an
    (n, n, n//2+1) complex64 array."""
    return c._pm_delta_k()


def force_mesh(axis):
    """Force mesh of one axis after compute_force, an (n, n, n) array."""
    return c._pm_force_mesh(axis)
