"""State: q, aux, t and problem_data on one patch (src/pyclaw/state.py:12-305).

q and aux keep the reference's shape and order, ``q[m, i, j]`` as Fortran-ordered
numpy arrays.  Once a ClawSolver2D is set up, the authoritative copy of q lives
in device memory; ``state.q`` then downloads it on access (one device-to-host
copy, only when the device copy changed) and any access or assignment marks the
host copy for upload before the next step.
"""
import copy

import numpy as np


class State(object):
    def __init__(self, geom, num_eqn, num_aux=0):
        from . import geometry
        if isinstance(geom, geometry.Patch):
            self.patch = geom
        elif isinstance(geom, geometry.Domain):
            self.patch = geom.patches[0]
        else:
            raise Exception("A PyClaw State object must be initialized with a PyClaw Patch object.")
        self.p = None
        self.F = None
        self.problem_data = {}
        self.t = 0.
        self.index_capa = -1
        self.keep_gauges = False
        self.gauge_data = []
        self._dev = None            # set by the solver: object with download()/host_changed()
        self._q = self.new_array(num_eqn)
        self._aux = self.new_array(num_aux)

    # ---- q / aux with device synchronisation ----------------------------
    @property
    def q(self):
        if self._dev is not None:
            self._dev.refresh_host_q(self)
            self._dev.host_q_touched()
        return self._q

    @q.setter
    def q(self, value):
        self._q = value
        if self._dev is not None:
            self._dev.host_q_assigned()

    @property
    def aux(self):
        if self._dev is not None:
            self._dev.host_aux_touched()
        return self._aux

    @aux.setter
    def aux(self, value):
        self._aux = value
        if self._dev is not None:
            self._dev.host_aux_touched()

    def get_q_host(self):
        """q on the host without marking it modified (read-only use)."""
        if self._dev is not None:
            self._dev.refresh_host_q(self)
        return self._q

    # ---- reference properties ------------------------------------------
    @property
    def num_eqn(self):
        if self._q is None:
            raise Exception('state.num_eqn has not been set.')
        return self._q.shape[0]

    @property
    def num_aux(self):
        return self._aux.shape[0] if self._aux is not None else 0

    @property
    def mp(self):
        return self.p.shape[0] if self.p is not None else 0

    @mp.setter
    def mp(self, mp):
        if self.p is not None:
            raise Exception('Cannot change state.mp after aux is initialized.')
        self.p = self.new_array(mp)

    @property
    def mF(self):
        return self.F.shape[0] if self.F is not None else 0

    @mF.setter
    def mF(self, mF):
        if self.F is not None:
            raise Exception('Cannot change state.mF after aux is initialized.')
        self.F = self.new_array(mF)

    @property
    def grid(self):
        return self.patch.grid

    def is_valid(self):
        return bool(self._q is not None and self._q.flags['F_CONTIGUOUS'])

    def set_cparam(self, fortran_module):
        """Kept for API compatibility: problem_data is read by the solver at setup."""
        pass

    def set_num_ghost(self, num_ghost):
        pass

    def new_array(self, dof):
        if dof == 0:
            return None
        shape = [dof]
        shape.extend(self.grid.num_cells)
        return np.empty(shape, order='F')

    def get_q_global(self):
        return self.get_q_host().copy()

    def get_aux_global(self):
        return self._aux.copy() if self._aux is not None else None

    def sum_F(self, i):
        return np.sum(np.abs(self.F[i, ...]))

    def __deepcopy__(self, memo={}):
        result = self.__class__(copy.deepcopy(self.patch), self.num_eqn, self.num_aux)
        result.t = self.t
        result._q = copy.deepcopy(self.get_q_host())
        if self._aux is not None:
            result._aux = copy.deepcopy(self._aux)
        result.problem_data = copy.deepcopy(self.problem_data)
        result.index_capa = self.index_capa
        return result

    def __str__(self):
        out = "PyClaw State object\nPatch dimensions: %s\nTime  t=%s\n" % (
            str(self.patch.num_cells_global), self.t)
        out += "Number of conserved quantities: %s\n" % str(self.num_eqn)
        if self._aux is not None:
            out += "Number of auxiliary fields: %s\n" % str(self.num_aux)
        if self.problem_data != {}:
            out += "problem_data: " + str(self.problem_data)
        return out
