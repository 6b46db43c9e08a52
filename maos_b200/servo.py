"""Device servo filter (``mb_servo_*``): ``lib/servo.c`` ``servo_new`` /
``servo_filter`` / ``servo_reset`` for batched DM commands on the GPU.

    s = Servo(n, ep=[[0.5]], ap=None, al=0, dt=1/800)
    cmd = s.filter(merr)          # torch CUDA float64 tensors of n values
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import native
from .native import check


class Servo:
    def __init__(self, n: int, ep, ap: Optional[np.ndarray] = None, al: int = 0, dt: float = 1 / 800,
                 device: int = 0):
        import torch
        self.lib = native.load()
        self.n = int(n)
        e = np.asfortranarray(np.atleast_2d(np.asarray(ep, dtype=np.float64)))
        a = None if ap is None else np.ascontiguousarray(ap, dtype=np.float64)
        h = C.c_void_p()
        check(self.lib.mb_servo_create(self.n, a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None,
                                       0 if a is None else len(a), int(al), e.ctypes.data_as(C.POINTER(C.c_double)),
                                       e.shape[0], e.shape[1], float(dt), C.byref(h)), "mb_servo_create")
        self.h = h
        self.cmd = torch.zeros(self.n, dtype=torch.float64, device=f"cuda:{device}")

    def filter(self, merr, stream=None):
        """One step; ``merr`` a CUDA float64 tensor of n values.  Returns the
        command tensor (kept by this object, overwritten by the next step)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream()
        check(self.lib.mb_servo_filter(self.h, C.c_void_p(merr.data_ptr()), C.c_void_p(self.cmd.data_ptr()),
                                       C.c_void_p(st.cuda_stream)), "mb_servo_filter")
        return self.cmd

    def reset(self):
        check(self.lib.mb_servo_reset(self.h), "mb_servo_reset")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_servo_free(self.h)
            self.h = None
