"""Rank queries (py/fs/comm.py).  One process drives one GPU: rank 0 of 1."""
from . import _fs as c


def this_node():
    """Returns the rank of this process (always 0)."""
    return c.comm_this_node()


def n_nodes():
    """Returns the number of processes in the run (always 1)."""
    return c.comm_n_nodes()
