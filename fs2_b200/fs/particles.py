"""Particle set (py/fs/particles.py), resident in GPU memory."""
from . import _fs as c


class Particles(object):
    """A set of particles.  Use fs.lpt.init() to create one with initial
    conditions, or Particles(np, boxsize) and append().

    Attributes (copied from the GPU on access):
        x, dx1, dx2, force, v (np.array float32, (np_local, 3)),
        id (np.array uint64), np_local, np_total.
    """

    def __init__(self, np=10, boxsize=0.0, *, _particles=None):
        if _particles is None:
            self._particles = c._particles_alloc(np, boxsize)
        else:
            self._particles = _particles

    def __getitem__(self, index):
        """particles[i] -> (x, y, z); particles[i:j:k] -> rows of
        x, v, dx1, dx2 and the id bytes, as a (n, 14) float32 array."""
        return c._particles_getitem(self._particles, index)

    def __len__(self):
        return c._particles_len(self._particles)

    def update_np_total(self):
        c._particles_update_np_total(self._particles)

    def append(self, x):
        """Appends particles with positions x, an (n, >=3) float64 array; None
        changes nothing."""
        c._particles_append(self._particles, x)

    def clear(self):
        """Removes all particles."""
        c._particles_clear(self._particles)

    def slice(self, frac):
        """Rows (as __getitem__) of particles with wrapped z < frac*boxsize."""
        return c._particles_slice(self._particles, frac)

    def periodic_wrapup(self):
        """Wraps positions into [0, boxsize)."""
        c._particles_periodic_wrapup(self._particles)

    def set(self, field, array):
        """Copies a host array into a field ('x', 'v', 'dx1', 'dx2', 'f' as
        (n, 3) float32, 'id' as (n,) uint64) and sets np_local = n."""
        c._particles_set(self._particles, field, array)

    @property
    def a(self):
        """(a_x, a_v, a_f): scale factors of positions, velocities, forces."""
        return c._particles_a(self._particles)

    def set_a(self, a_x, a_v, a_f):
        c._particles_a(self._particles, a_x, a_v, a_f)

    @property
    def boxsize(self):
        return c._particles_boxsize(self._particles)

    @property
    def np_local(self):
        return c._particles_len(self._particles)

    @property
    def np_total(self):
        return c._particles_np_total(self._particles)

    @property
    def id(self):
        return c._particles_id_asarray(self._particles)

    @property
    def x(self):
        return c._particles_x_asarray(self._particles, 0)

    @property
    def dx1(self):
        return c._particles_x_asarray(self._particles, 1)

    @property
    def dx2(self):
        return c._particles_x_asarray(self._particles, 2)

    @property
    def v(self):
        return c._particles_v_asarray(self._particles)

    @property
    def force(self):
        return c._particles_force_asarray(self._particles)

    def save_hdf5(self, filename, var):
        """Writes a snapshot (py/fs/particles.py:91-104,
        py/hdf5_write.cpp:28-187).

        Args:
            filename (str): Output file name.
            var (str): Output variables, a subset of 'ixvcf12' in this order:
                i: ID, x: positions, v: velocities (COLA's internal ones),
                c: velocities with the 2LPT part restored (written as 'v'),
                f: force, 1: 1LPT displacements, 2: 2LPT displacements.

        The datasets are those of the reference: 'id' (uint64), 'x', 'v',
        'f', 'dx1', 'dx2' ((np, 3) float32), and the scalars
        parameters/boxsize, omega_m, ax, av (float64) and parameters/nc
        (int32).  With h5py installed they are written as an HDF5 file;
        without it, into a NumPy .npz archive at `filename` with the same
        names ('parameters/boxsize' and so on), readable with numpy.load.
        """
        data = snapshot_datasets(self, var)
        try:
            import h5py
        except ImportError:
            h5py = None
        if h5py is not None:
            with h5py.File(filename, "a") as f:
                for name, arr in data.items():
                    if name in f:
                        del f[name]
                    f.create_dataset(name, data=arr)
            return
        import numpy as np
        with open(filename, "wb") as fh:
            np.savez(fh, **data)


def snapshot_datasets(particles, var):
    """The datasets save_hdf5 writes for `var` (a subset of 'ixvcf12' in
    that order; anything left over is an error, as in
    py/hdf5_write.cpp:132-135)."""
    import ctypes
    import math
    import numpy as np
    from . import cola
    from .. import capi
    om = ctypes.c_double()
    capi.call("fs2g_cosmology_omega_m", ctypes.byref(om))
    a_x, a_v, _ = particles.a
    nc = int(round(math.pow(float(particles.np_total), 1.0 / 3.0)))
    out = {
        "parameters/boxsize": np.float64(particles.boxsize),
        "parameters/omega_m": np.float64(om.value),
        "parameters/ax": np.float64(a_x),
        "parameters/av": np.float64(a_v),
        "parameters/nc": np.int32(nc),
    }
    fields = (("i", "id", lambda: particles.id),
              ("x", "x", lambda: particles.x),
              ("v", "v", lambda: particles.v),
              ("c", "v", lambda: cola.velocity(particles)),
              ("f", "f", lambda: particles.force),
              ("1", "dx1", lambda: particles.dx1),
              ("2", "dx2", lambda: particles.dx2))
    rest = var
    for key, name, get in fields:
        if rest[:1] == key:
            out[name] = get()
            rest = rest[1:]
    if rest:
        raise ValueError("unknown option for hdf5_write, %s" % rest)
    return out
