"""vamtoolbox.util.timing (vamtoolbox/util/timing.py:4-19)."""
import functools
import time


def timing(func):
    """Decorator printing the wall time of each call of func."""

    @functools.wraps(func)
    def wrap(*args, **kwargs):
        t0 = time.time()
        ret = func(*args, **kwargs)
        print("%s function took %0.4f seconds" % (func.__name__, time.time() - t0))
        return ret

    return wrap
