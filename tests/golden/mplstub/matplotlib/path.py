"""Import stub for matplotlib.path (plotting is not used by the BEM path)."""


class Path(object):
    def __init__(self, *args, **kwargs):
        raise RuntimeError("matplotlib.path is stubbed out for fixture generation")
