"""Device-resident state of one ClawSolver2D: buffers held as torch tensors,
kernels launched through the C ABI of libclaw2.so on torch's current stream.

Buffers (device layout of include/claw2.h, ghost cells included):
  q[0], q[1]  ping-pong state buffers; control.cur says which one is current
  aux         auxiliary fields, ghost cells filled once per upload
  scratch     per-CTA CFL partials + block-arrival counter
  ctrl        claw2_control (device-side time-step controller)
"""
import ctypes

import numpy as np

from . import _abi
from . import _lib


def _torch():
    import torch
    return torch


class DeviceState(object):
    def __init__(self, problem, device=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise _lib.ClawLibraryError("pyclaw_b200 needs a CUDA device (sm_100a); none is available")
        self.lib = _lib.load()
        self.p = problem
        _lib.check(self.lib.claw2_validate(ctypes.byref(problem)), "claw2_validate")
        self.L = _lib.layout(problem)
        self.device = torch.device(device if device is not None else "cuda")
        f64 = dict(dtype=torch.float64, device=self.device)
        self.q = [torch.zeros(self.L.q_elems, **f64), torch.zeros(self.L.q_elems, **f64)]
        self.aux = torch.zeros(max(self.L.aux_elems, 1), **f64)
        nscr = int(self.lib.claw2_scratch_bytes(ctypes.byref(problem)))
        self.scratch = torch.zeros((nscr + 7) // 8 * 8, dtype=torch.uint8, device=self.device)
        self.ctrl = torch.zeros(ctypes.sizeof(_abi.Control), dtype=torch.uint8, device=self.device)
        self.ctrl_host = torch.zeros(ctypes.sizeof(_abi.Control), dtype=torch.uint8).pin_memory()
        self.cfl_dev = torch.zeros(1, **f64)
        self.cur = 0
        self.device_newer = False       # device q changed since the last download
        self.host_dirty = True          # host q may differ from the device copy
        self.aux_dirty = True
        self.state = None

    # ---- plumbing ----------------------------------------------------------
    @property
    def stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream(self.device).cuda_stream)

    def ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def qview(self, k):
        return self.q[k].view(self.p.num_eqn, self.L.rows, self.L.ld)

    def interior(self, k):
        g = _abi.NUM_GHOST
        return self.qview(k)[:, g:g + self.p.my, g:g + self.p.mx]

    # ---- host <-> device -------------------------------------------------
    def attach(self, state):
        self.state = state
        state._dev = self

    def host_q_touched(self):
        self.host_dirty = True

    def host_q_assigned(self):
        """state.q was replaced on the host: the host copy is now authoritative."""
        self.host_dirty = True
        self.device_newer = False

    def host_aux_touched(self):
        self.aux_dirty = True

    def refresh_host_q(self, state):
        if self.device_newer:
            state._q = self.download_q()
            self.device_newer = False

    def download_q(self):
        v = self.interior(self.cur).permute(0, 2, 1).cpu().numpy()
        return np.asfortranarray(v)

    def upload_q(self, q):
        torch = _torch()
        src = torch.from_numpy(np.ascontiguousarray(np.asarray(q, dtype=np.float64).transpose(0, 2, 1)))
        self.interior(self.cur).copy_(src)
        _lib.check(self.lib.claw2_fill_ghosts(ctypes.byref(self.p), self.ptr(self.q[self.cur]), self.stream),
                   "claw2_fill_ghosts")

    def upload_aux(self, aux):
        if self.p.num_aux == 0:
            return
        torch = _torch()
        g = _abi.NUM_GHOST
        v = self.aux[:self.L.aux_elems].view(self.p.num_aux, self.L.rows, self.L.ld)
        src = torch.from_numpy(np.ascontiguousarray(np.asarray(aux, dtype=np.float64).transpose(0, 2, 1)))
        v[:, g:g + self.p.my, g:g + self.p.mx].copy_(src)
        _lib.check(self.lib.claw2_fill_aux_ghosts(ctypes.byref(self.p), self.ptr(self.aux), self.stream),
                   "claw2_fill_aux_ghosts")

    def sync_from_host(self):
        """Upload whatever the host side may have changed since the last step."""
        st = self.state
        if self.aux_dirty:
            if st._aux is not None:
                self.upload_aux(st._aux)
            self.aux_dirty = False
        if self.host_dirty:
            self.upload_q(st._q)
            self.host_dirty = False
            self.device_newer = False

    def cells_q(self, cells):
        """q(:, ix, iy) of the current state at the interior cells `cells`,
        gathered on the device (one small copy instead of the whole field)."""
        torch = _torch()
        ix = torch.tensor([c[0] for c in cells], dtype=torch.long, device=self.device)
        iy = torch.tensor([c[1] for c in cells], dtype=torch.long, device=self.device)
        return self.interior(self.cur)[:, iy, ix].cpu().numpy()

    def ghosted_ref(self):
        """Current q with ghost cells, in the reference layout (num_eqn, mx+4, my+4), on the host."""
        v = self.qview(self.cur)[:, :, :self.p.mx + 2 * _abi.NUM_GHOST].permute(0, 2, 1).cpu().numpy()
        return np.asfortranarray(v)

    def set_ghosted_ref(self, qbc, k=None):
        torch = _torch()
        k = self.cur if k is None else k
        src = torch.from_numpy(np.ascontiguousarray(np.asarray(qbc).transpose(0, 2, 1)))
        self.qview(k)[:, :, :self.p.mx + 2 * _abi.NUM_GHOST].copy_(src)

    # ---- stepping ---------------------------------------------------------
    def step(self, dt):
        """One step q[cur] -> q[1-cur] with explicit dt; returns the CFL number."""
        nxt = 1 - self.cur
        _lib.check(self.lib.claw2_step(ctypes.byref(self.p), self.ptr(self.q[self.cur]), self.ptr(self.q[nxt]),
                                       self.ptr(self.aux), float(dt), self.ptr(self.scratch),
                                       self.ptr(self.cfl_dev), self.stream), "claw2_step")
        cfl = float(self.cfl_dev.item())
        return cfl, nxt

    def gauge_recorder(self, cells, capacity):
        """Device buffers of a claw2_gauges recorder for the interior cells
        `cells` [(ix, iy), ...]; rows are drained by evolve()."""
        torch = _torch()
        g = _abi.Gauges()
        n = len(cells)
        self._g_cells = torch.tensor([c for xy in cells for c in xy], dtype=torch.int32, device=self.device)
        self._g_record = torch.zeros(capacity * n * (1 + self.p.num_eqn), dtype=torch.float64, device=self.device)
        self._g_state = torch.zeros(3, dtype=torch.int64, device=self.device)
        g.ngauges, g.capacity = n, capacity
        g.cells, g.record, g.state = (self._g_cells.data_ptr(), self._g_record.data_ptr(), self._g_state.data_ptr())
        return g

    def evolve(self, control, max_batch=256, hooks=None, gauges=None, on_gauges=None):
        """Run the device-controlled loop until control is done; returns the
        final Control.  hooks: a claw2_hooks (source term run on the device).
        gauges: a list of interior cells (ix, iy) sampled after every accepted
        step on the device; on_gauges(rows) gets the samples after every batch
        of steps, rows[r, k] = (t, q(:, ix_k, iy_k)) in step order."""
        torch = _torch()
        control.cur = self.cur
        host = _abi.Control.from_address(self.ctrl_host.data_ptr())
        ctypes.memmove(ctypes.addressof(host), ctypes.addressof(control), ctypes.sizeof(control))
        self.ctrl.copy_(self.ctrl_host, non_blocking=True)
        stream = torch.cuda.current_stream(self.device)
        rec = None
        if gauges:
            rec = self.gauge_recorder(gauges, max_batch)
            self._g_state[1] = int(control.numsteps)
        # each batch is the controller's estimate of the steps left (the
        # host reads the controller only between batches; steps launched
        # after it is done return at once)
        def estimate():
            left = max(1, int(host.max_steps - host.iter))       # loop iterations the controller allows
            if host.dt > 0:
                left = min(left, (host.tend - host.t) / host.dt + 1)
            return int(max(1, min(max_batch, left)))
        batch = estimate()
        while True:
            if rec is not None:
                _lib.check(self.lib.claw2_advance_gauged(ctypes.byref(self.p), self.ptr(self.q[0]),
                                                         self.ptr(self.q[1]), self.ptr(self.aux), self.ptr(self.ctrl),
                                                         self.ptr(self.scratch), int(batch),
                                                         ctypes.byref(hooks) if hooks is not None else None,
                                                         ctypes.byref(rec), self.stream), "claw2_advance_gauged")
                st = self._g_state.cpu()             # waits for the batch
                nrows = int(st[0])
                if int(st[2]):
                    raise RuntimeError("gauge recorder overflow")
                if nrows:
                    rows = self._g_record[:nrows * len(gauges) * (1 + self.p.num_eqn)].cpu().numpy()
                    self._g_state[0] = 0
                    if on_gauges is not None:
                        on_gauges(rows.reshape(nrows, len(gauges), 1 + self.p.num_eqn))
            elif hooks is None:
                _lib.check(self.lib.claw2_advance(ctypes.byref(self.p), self.ptr(self.q[0]), self.ptr(self.q[1]),
                                                  self.ptr(self.aux), self.ptr(self.ctrl), self.ptr(self.scratch),
                                                  int(batch), self.stream), "claw2_advance")
            else:
                _lib.check(self.lib.claw2_advance_hooked(ctypes.byref(self.p), self.ptr(self.q[0]),
                                                         self.ptr(self.q[1]), self.ptr(self.aux), self.ptr(self.ctrl),
                                                         self.ptr(self.scratch), int(batch), ctypes.byref(hooks),
                                                         self.stream), "claw2_advance_hooked")
            self.ctrl_host.copy_(self.ctrl, non_blocking=True)
            stream.synchronize()
            if host.done:
                break
            batch = estimate()
        out = _abi.Control()
        ctypes.memmove(ctypes.addressof(out), ctypes.addressof(host), ctypes.sizeof(out))
        self.cur = out.cur
        self.device_newer = True
        return out
