"""Controller.run: output times, frames and the evolve loop
(src/pyclaw/controller.py:20-316).  Frames are copied to the host only at
output times; the steps in between stay on the GPU."""
import copy
import logging
import os

import numpy as np

from .solver import Solver


class FrameCounter(object):
    def __init__(self):
        self.__frame = 0

    def get_counter(self):
        return self.__frame

    def increment(self):
        self.__frame += 1

    def set_counter(self, new_frame_num):
        self.__frame = new_frame_num

    def __repr__(self):
        return str(self.__frame)


class Controller(object):
    def __init__(self):
        self.xdir = os.getcwd()
        self.rundir = os.getcwd()
        self.outdir = os.getcwd() + '/_output'
        self.overwrite = True
        self.start_frame = 0
        self.solution = None
        self.solver = None
        self.keep_copy = False
        self.frames = []
        self.write_aux_init = False
        self.write_aux_always = False
        self.output_format = 'ascii'
        self.output_file_prefix = None
        self.output_options = {}
        self.tfinal = 1.0
        self.output_style = 1
        self.verbosity = 0
        self.num_output_times = 10
        self.out_times = np.linspace(0.0, self.tfinal, self.num_output_times - self.start_frame)
        self.nstepout = 1
        self.compute_p = None
        self.file_prefix_p = 'claw_p'
        self.compute_F = None
        self.F_file_name = 'F'
        self.logger = logging.getLogger('pyclaw.controller')

    outdir_p = property(lambda self: os.path.join(self.outdir, '_p'))
    F_path = property(lambda self: os.path.join(self.outdir, self.F_file_name + '.txt'))

    def check_validity(self):
        if self.solver is None:
            raise Exception("No solver set in controller.")
        if not isinstance(self.solver, Solver):
            raise Exception("Solver is not of correct type.")
        if not self.solver.is_valid():
            raise Exception("The solver failed to initialize properly.")
        if not self.solution.is_valid():
            raise Exception("Initial solution is not valid.")

    def run(self):
        self.start_frame = self.solution.start_frame
        if len(self.solution.patch.grid.gauges) > 0:
            self.solution.patch.grid.setup_gauge_files(self.outdir)
        frame = FrameCounter()
        frame.set_counter(self.start_frame)
        if self.keep_copy:
            self.frames = []
        self.solver.setup(self.solution)
        self.solver.dt = self.solver.dt_initial
        self.check_validity()
        self.solver.write_gauge_values(self.solution)
        if self.output_style == 1:
            output_times = np.linspace(self.solution.t, self.tfinal, self.num_output_times + 1 - self.start_frame)
        elif self.output_style == 2:
            output_times = self.out_times
        elif self.output_style == 3:
            output_times = np.ones((self.num_output_times + 1 - self.start_frame))
        else:
            raise Exception("Invalid output style %s" % self.output_style)
        if self.keep_copy:
            self.frames.append(copy.deepcopy(self.solution))
        if self.output_format is not None:
            if os.path.exists(self.outdir) and self.overwrite is False:
                raise Exception("Refusing to overwrite existing output data. "
                                "\nEither delete/move the directory or set controller.overwrite=True.")
            self.solution.write(frame, self.outdir, self.output_format, self.output_file_prefix,
                                self.write_aux_init, self.output_options)
        status = None
        for t in output_times[1:]:
            if self.output_style < 3:
                status = self.solver.evolve_to_time(self.solution, t)
            else:
                for n in range(self.nstepout):
                    status = self.solver.evolve_to_time(self.solution)
            frame.increment()
            if self.keep_copy:
                self.frames.append(copy.deepcopy(self.solution))
            if self.output_format is not None:
                self.solution.write(frame, self.outdir, self.output_format, self.output_file_prefix,
                                    self.write_aux_always, self.output_options)
            self.logger.info("Solution %s computed for time t=%f" % (frame, self.solution.t))
            for gfile in self.solution.state.grid.gauge_files:
                gfile.flush()
        self.solver.teardown()
        for gfile in self.solution.state.grid.gauge_files:
            gfile.close()
        return status
