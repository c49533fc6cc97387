class Inert(object):
    """A value on which any attribute access, call or arithmetic returns another Inert."""
    def __getattr__(self, name):
        if name.startswith('__'):
            raise AttributeError(name)
        return Inert()

    def __call__(self, *args, **kwargs):
        return Inert()

    def _op(self, *args):
        return Inert()

    __mul__ = __rmul__ = __truediv__ = __rtruediv__ = __pow__ = __add__ = __radd__ = _op
    __sub__ = __rsub__ = __neg__ = _op

    def __eq__(self, other):
        return self is other

    def __hash__(self):
        return id(self)
