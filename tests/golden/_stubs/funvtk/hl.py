def gridToVTK(*args, **kwargs):
    pass


def pointsToVTK(*args, **kwargs):
    pass
