"""Host-resident batches through the GPU with copies and compute overlapped.

A batch of wave functions that lives in (pinned) host memory is processed
in chunks of bands: while chunk i is computed, chunk i+1 is copied in and
chunk i-1 is copied out, on three streams (copy-in, compute, copy-out) with
two sets of device buffers.  Host-to-device and device-to-host copies use
different copy engines, so the wall time approaches the larger of the two
transfer volumes instead of their sum plus the compute.

``StepPipeline`` runs the finite-difference step of a band batch: the
kinetic operator applied to every band, and the restriction of every band
to the coarse grid followed by its interpolation back (the operations of
gpaw/fd_operators.py:120-130 and gpaw/transformers.py:79-91).  Results are
identical to running the same operators on the whole batch at once (every
band is computed the same way in any chunk).
"""
from __future__ import annotations

import torch


class StepPipeline:
    def __init__(self, kin, rst, itp, chunk=32, device=None):
        self.kin, self.rst, self.itp = kin, rst, itp
        self.chunk = int(chunk)
        self.device = torch.device(device if device is not None else 'cuda')
        self.s_in = torch.cuda.Stream(device=self.device)
        self.s_run = torch.cuda.Stream(device=self.device)
        self.s_out = torch.cuda.Stream(device=self.device)
        self._bufs = None

    def _buffers(self, fine, coarse, dtype):
        key = (fine, coarse, dtype)
        if self._bufs is None or self._bufs[0] != key:
            mk = lambda shape: torch.empty((self.chunk,) + shape, dtype=dtype,
                                           device=self.device)
            sets = [{'x': mk(fine), 'y': mk(fine), 'c': mk(coarse),
                     'z': mk(fine)} for _ in range(2)]
            self._bufs = (key, sets)
        return self._bufs[1]

    def run(self, host_in, host_y, host_c, host_z, phases=None):
        """host_in -> host_y = kin(host_in), host_c = restrict(host_in),
        host_z = interpolate(host_c); all host tensors (pinned for the
        copies to overlap), bands along the first axis.  Returns when the
        results are in host memory."""
        nb = host_in.shape[0]
        fine = tuple(host_in.shape[1:])
        coarse = tuple(host_c.shape[1:])
        bufs = self._buffers(fine, coarse, host_in.dtype)
        cur = torch.cuda.current_stream(self.device)
        for s in (self.s_in, self.s_run, self.s_out):
            s.wait_stream(cur)
        free = [None, None]      # copy-out done: buffer set reusable
        for i, b0 in enumerate(range(0, nb, self.chunk)):
            k = i % 2
            n = min(self.chunk, nb - b0)
            B = bufs[k]
            x, y, c, z = (B[t][:n] for t in 'xycz')
            with torch.cuda.stream(self.s_in):
                if free[k] is not None:
                    self.s_in.wait_event(free[k])
                x.copy_(host_in[b0:b0 + n], non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(ev_in)
                self.kin.apply(x, y, phases)
                self.rst.apply(x, c, phases=phases)
                self.itp.apply(c, z, phases=phases)
                ev_run = torch.cuda.Event()
                ev_run.record(self.s_run)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(ev_run)
                host_y[b0:b0 + n].copy_(y, non_blocking=True)
                host_c[b0:b0 + n].copy_(c, non_blocking=True)
                host_z[b0:b0 + n].copy_(z, non_blocking=True)
                ev_out = torch.cuda.Event()
                ev_out.record(self.s_out)
                free[k] = ev_out
        self.s_out.synchronize()
