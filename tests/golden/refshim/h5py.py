"""No-op stand-in for ``h5py`` so ``set_simulator`` imports; nothing is written."""


class _Group(dict):
    def __init__(self):
        super().__init__()
        self.attrs = {}

    def create_dataset(self, *a, **k):
        return None


class File(dict):
    def __init__(self, *a, **k):
        super().__init__()

    def create_group(self, key):
        g = _Group()
        self[key] = g
        return g

    def close(self):
        pass
