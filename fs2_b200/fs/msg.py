"""Log level (py/fs/msg.py)."""
from . import _fs as c

dict_loglevel = {'debug': 0, 'verbose': 1, 'info': 2, 'warn': 3, 'error': 4,
                 'fatal': 5}


def set_loglevel(loglevel):
    """Sets the amount of messages: an int 0-5 or one of the names of
    dict_loglevel."""
    if isinstance(loglevel, str):
        loglevel = dict_loglevel[loglevel]
    c.set_loglevel(loglevel)
