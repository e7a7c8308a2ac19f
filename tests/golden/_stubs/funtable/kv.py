"""No-op ``SQLiteStore`` stand-in: the reference logs every step to SQLite."""


class _Table:
    def set(self, *args, **kwargs):
        pass


class SQLiteStore:
    def __init__(self, *args, **kwargs):
        pass

    def create_kv_table(self, *args, **kwargs):
        pass

    def create_kkv_table(self, *args, **kwargs):
        pass

    def get_table(self, *args, **kwargs):
        return _Table()
