"""``funutil.cache.cache`` stand-in: a pass-through decorator.  The reference
only applies it to pure functions, so skipping memoisation keeps results."""


def cache(fn=None, *args, **kwargs):
    if fn is None or not callable(fn):
        return lambda f: f
    return fn
