"""CompStruct: wavelength-tagged bag of fields on a particle surface.

Same access patterns as the reference's ``CompStruct``
(mnpbem/greenfun/compgreen_stat.py:1154-1275): attribute and item access to
the fields, ``.p``, ``.enei``, ``get`` with default and ``set``.
"""


class CompStruct(object):
    def __init__(self, p, enei=None, **fields):
        object.__setattr__(self, 'p', p.p if isinstance(p, CompStruct) else p)
        object.__setattr__(self, 'enei', p.enei if isinstance(p, CompStruct) else enei)
        object.__setattr__(self, 'val', dict(p.val) if isinstance(p, CompStruct) else {})
        self.val.update(fields)

    def __getattr__(self, name):
        val = object.__getattribute__(self, 'val')
        if name in val:
            return val[name]
        raise AttributeError("'CompStruct' object has no attribute '{}'".format(name))

    def __setattr__(self, name, value):
        if name in ('p', 'enei', 'val'):
            object.__setattr__(self, name, value)
        else:
            self.val[name] = value

    def __getitem__(self, key):
        if key == 'p':
            return self.p
        if key == 'enei':
            return self.enei
        return self.val[key]

    def __setitem__(self, key, value):
        setattr(self, key, value)

    def __contains__(self, key):
        return key in self.val

    def get(self, key, default=None):
        try:
            return self[key]
        except KeyError:
            return default

    def set(self, **fields):
        self.val.update(fields)
        return self
