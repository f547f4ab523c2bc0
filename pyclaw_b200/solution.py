"""Solution: the states of a domain at one time (src/pyclaw/solution.py).

Solution(state, domain) wraps a State; Solution(frame, path=..., file_format=
'ascii', read_aux=...) reads a frame written by Solution.write (restart).
"""
import copy
import os


class Solution(object):
    def __init__(self, *arg, **kargs):
        from .geometry import Domain, Patch, Dimension
        from .state import State
        self.states = []
        self.domain = None
        self._start_frame = 0
        if len(arg) == 1 and isinstance(arg[0], int) or (len(arg) >= 1 and isinstance(arg[0], int)):
            frame = arg[0]
            self.read(frame, **kargs)
            return
        if len(arg) == 0:
            return
        if isinstance(arg[0], State):
            self.states = [arg[0]]
        elif isinstance(arg[0], (list, tuple)) and len(arg[0]) and isinstance(arg[0][0], State):
            self.states = list(arg[0])
        if len(arg) > 1:
            self.domain = arg[1]
        elif self.states:
            self.domain = Domain(self.states[0].patch)
        del Patch, Dimension

    # reference properties (solution.py:24-100)
    state = property(lambda self: self.states[0])
    patch = property(lambda self: self.states[0].patch)
    num_eqn = property(lambda self: self.states[0].num_eqn)
    num_aux = property(lambda self: self.states[0].num_aux)
    start_frame = property(lambda self: self._start_frame)

    @property
    def t(self):
        return self.states[0].t

    @t.setter
    def t(self, value):
        for s in self.states:
            s.t = value

    def is_valid(self):
        return all(s.is_valid() for s in self.states)

    def write(self, frame, path='./', file_format='ascii', file_prefix=None, write_aux=False,
              options={}, write_p=False):
        """Write the frame (solution.py:247-296); ascii is supported."""
        from .io import ascii as _ascii
        if not os.path.exists(path):
            os.makedirs(path)
        formats = [file_format] if isinstance(file_format, str) else list(file_format)
        for fmt in formats:
            if fmt != 'ascii':
                raise NotImplementedError("output format %s is not built; use 'ascii'" % fmt)
            _ascii.write(self, frame, path, file_prefix or 'fort', write_aux, options, write_p)

    def read(self, frame, path='./_output', file_format='ascii', file_prefix=None, read_aux=True,
             options={}, **kargs):
        from .io import ascii as _ascii
        if file_format != 'ascii':
            raise NotImplementedError("input format %s is not built; use 'ascii'" % file_format)
        _ascii.read(self, frame, path, file_prefix or 'fort', read_aux, options)
        self._start_frame = frame

    def __deepcopy__(self, memo={}):
        result = self.__class__()
        result.states = [copy.deepcopy(s) for s in self.states]
        result.domain = copy.deepcopy(self.domain)
        result._start_frame = self._start_frame
        return result
