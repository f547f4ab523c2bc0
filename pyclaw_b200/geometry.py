"""Grid geometry: Dimension, Grid, Patch, Domain.

Same constructors and attributes as the reference (src/pyclaw/geometry.py):
Dimension('x', lower, upper, num_cells) or Dimension(lower, upper, num_cells,
name='x'); delta = (upper-lower)/num_cells (:425-427); centers[i] =
lower + (i+0.5)*delta and edges[i] = lower + i*delta, computed element by
element as the reference does so that initial data built on them is
bit-identical (:429-446).
"""
import copy

import numpy as np


def default_mapc2p(patch, x):
    return x


class Dimension(object):
    def __init__(self, *args, **kargs):
        self.name = 'x'
        self.num_cells = None
        self.lower = 0.0
        self.upper = 1.0
        self.on_lower_boundary = None
        self.on_upper_boundary = None
        self.units = None
        if isinstance(args[0], (float, int)) and not isinstance(args[0], bool) and len(args) >= 3 \
                and not isinstance(args[0], str):
            self.lower = float(args[0])
            self.upper = float(args[1])
            self.num_cells = int(args[2])
        elif isinstance(args[0], str):
            self.name = args[0]
            self.lower = float(args[1])
            self.upper = float(args[2])
            self.num_cells = int(args[3])
        else:
            raise Exception("Invalid initializer for Dimension.")
        for k, v in kargs.items():
            setattr(self, k, v)
        self._edges = None
        self._centers = None

    @property
    def delta(self):
        return (self.upper - self.lower) / float(self.num_cells)

    @property
    def edges(self):
        if self._edges is None:
            self._edges = np.empty(self.num_cells + 1)
            for i in range(self.num_cells + 1):
                self._edges[i] = self.lower + i * self.delta
        return self._edges

    @property
    def centers(self):
        if self._centers is None:
            self._centers = np.empty(self.num_cells)
            for i in range(self.num_cells):
                self._centers[i] = self.lower + (i + 0.5) * self.delta
        return self._centers

    def centers_with_ghost(self, nghost):
        centers = self.centers
        pre = np.linspace(self.lower - (nghost - 0.5) * self.delta, self.lower - 0.5 * self.delta, nghost)
        post = np.linspace(self.upper + 0.5 * self.delta, self.upper + (nghost - 0.5) * self.delta, nghost)
        return np.hstack((pre, centers, post))

    def __str__(self):
        out = "Dimension %s" % self.name
        if self.units:
            out += " (%s)" % self.units
        return out + ":  (num_cells,delta,[lower,upper]) = (%s,%s,[%s,%s])" % (
            self.num_cells, self.delta, self.lower, self.upper)


class Grid(object):
    """Dimensions plus per-dimension attribute lists (geometry.py:23-335)."""

    def __init__(self, dimensions):
        self.mapc2p = default_mapc2p
        self.gauges = []
        self.gauge_file_names = []
        self.gauge_files = []
        self.gauge_dir_name = '_gauges'
        if isinstance(dimensions, Dimension):
            dimensions = [dimensions]
        self._dimensions = []
        for dim in dimensions:
            self.add_dimension(dim)

    def __getattr__(self, key):
        if key in ('num_cells', 'lower', 'upper', 'delta', 'units', 'centers', 'edges',
                   'on_lower_boundary', 'on_upper_boundary'):
            return self.get_dim_attribute(key)
        raise AttributeError("'Grid' object has no attribute '" + key + "'")

    @property
    def num_dim(self):
        return len(self._dimensions)

    @property
    def dimensions(self):
        return [getattr(self, name) for name in self._dimensions]

    def add_dimension(self, dimension):
        if dimension.name in self._dimensions:
            raise Exception('Unable to add dimension. A dimension of the same name: %s, already exists.'
                            % dimension.name)
        self._dimensions.append(dimension.name)
        setattr(self, dimension.name, dimension)

    def get_dim_attribute(self, attr):
        return [getattr(dim, attr) for dim in self.dimensions]

    @property
    def c_centers(self):
        """Computational cell centres, one meshgrid array per dimension."""
        return list(np.meshgrid(*self.get_dim_attribute('centers'), indexing='ij'))

    @property
    def p_centers(self):
        return self.mapc2p(self, self.c_centers)

    @property
    def c_edges(self):
        return list(np.meshgrid(*self.get_dim_attribute('edges'), indexing='ij'))

    def add_gauges(self, gauge_coords):
        """Record the cell indices of gauge points (geometry.py:336-356)."""
        for gauge in gauge_coords:
            if all(self.lower[n] <= gauge[n] < self.upper[n] for n in range(self.num_dim)):
                idx = [int(round((gauge[n] - self.lower[n]) / self.delta[n])) for n in range(self.num_dim)]
                self.gauges.append(idx)
                self.gauge_file_names.append('gauge' + '_'.join(str(c) for c in gauge) + '.txt')

    def setup_gauge_files(self, outdir):
        import os
        gdir = os.path.join(outdir, self.gauge_dir_name)
        os.makedirs(gdir, exist_ok=True)
        self.gauge_files = [open(os.path.join(gdir, n), 'a') for n in self.gauge_file_names]

    def __str__(self):
        return '\n'.join(str(d) for d in self.dimensions)


class Patch(object):
    """A logically rectangular patch (geometry.py:507-597)."""

    def __init__(self, dimensions):
        self.level = 1
        self.patch_index = 1
        if isinstance(dimensions, Dimension):
            dimensions = [dimensions]
        self._dimensions = []
        for dim in dimensions:
            dim.on_lower_boundary = True
            dim.on_upper_boundary = True
            self.add_dimension(dim)
        self.grid = Grid(dimensions)

    num_cells_global = property(lambda self: self.get_dim_attribute('num_cells'))
    lower_global = property(lambda self: self.get_dim_attribute('lower'))
    upper_global = property(lambda self: self.get_dim_attribute('upper'))
    num_dim = property(lambda self: len(self._dimensions))
    dimensions = property(lambda self: [getattr(self, n) for n in self._dimensions])
    delta = property(lambda self: self.get_dim_attribute('delta'))
    name = property(lambda self: self._dimensions)

    def add_dimension(self, dimension):
        if dimension.name in self._dimensions:
            raise Exception('Unable to add dimension. A dimension of the same name: %s, already exists.'
                            % dimension.name)
        self._dimensions.append(dimension.name)
        setattr(self, dimension.name, dimension)

    def get_dim_attribute(self, attr):
        return [getattr(getattr(self, name), attr) for name in self._dimensions]

    def __deepcopy__(self, memo={}):
        result = self.__class__(copy.deepcopy(self.dimensions))
        result.level = self.level
        result.patch_index = self.patch_index
        return result

    def __str__(self):
        return "Patch %s:\n" % self.patch_index + '\n'.join(str(d) for d in self.dimensions)


class Domain(object):
    """A list of patches (geometry.py:600-667)."""

    def __init__(self, *arg):
        if len(arg) > 1:
            lower, upper, n = arg[0], arg[1], arg[2]
            names = ['x', 'y', 'z'][:len(n)]
            dims = [Dimension(lo, up, nn, name=nm) for lo, up, nn, nm in zip(lower, upper, n, names)]
            self.patches = [Patch(dims)]
        else:
            geom = arg[0]
            if not isinstance(geom, (list, tuple)):
                geom = [geom]
            if isinstance(geom[0], Patch):
                self.patches = list(geom)
            elif isinstance(geom[0], Dimension):
                self.patches = [Patch(geom)]

    num_dim = property(lambda self: self.patches[0].num_dim)
    patch = property(lambda self: self.patches[0])
    grid = property(lambda self: self.patches[0].grid)

    def __deepcopy__(self, memo={}):
        return self.__class__(copy.deepcopy(self.patches))
