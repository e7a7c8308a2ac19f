"""Minimal stand-in for the absent ``funutil`` package (pinned 1.0.48 by the
reference's lock file).  Only what funlbm imports is provided: ``deep_get``,
``run_timer``, ``getLogger`` and ``funutil.cache.cache``.  Used only when the
golden-fixture script imports the reference; never by the product."""
import functools


def deep_get(obj, key, default=None):
    """Look up ``key`` in a dict; dotted keys walk nested dicts."""
    if obj is None:
        return default
    cur = obj
    for part in str(key).split("."):
        if isinstance(cur, dict) and part in cur:
            cur = cur[part]
        else:
            return default
    return cur


def run_timer(fn):
    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        return fn(*args, **kwargs)

    return wrapper


class _Logger:
    def __init__(self, name):
        self.name = name

    def _log(self, *args, **kwargs):
        pass

    info = error = success = warning = debug = _log


def getLogger(name="funutil"):
    return _Logger(name)
