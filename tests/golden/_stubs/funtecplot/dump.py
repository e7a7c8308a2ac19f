class PointData:
    def __init__(self, *args, **kwargs):
        pass

    def dump(self, *args, **kwargs):
        pass
