"""The learned part: the per-bead tensor-core network (cr_mlp_* in the C ABI)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

FEATURES = 48
HIDDEN = 128
NPARAM = 22913


class Network:
    """48 -> 128 -> 128 -> 1 GELU network; BF16 tcgen05 forward/backward, FP32 Adam."""

    def __init__(self, seed: int = 1):
        import torch

        self.torch = torch
        self.h = C.c_void_p()
        _lib.check(_lib.lib().cr_mlp_create(C.c_uint64(seed), C.byref(self.h)), "cr_mlp_create")

    def close(self):
        if self.h:
            _lib.lib().cr_mlp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, where):
        if st != _lib.CR_OK:
            msg = _lib.lib().cr_mlp_last_error(self.h)
            raise _lib.CrError(st, where, msg.decode() if msg else "")

    @staticmethod
    def _stream():
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def params(self) -> np.ndarray:
        p = np.zeros(NPARAM, dtype=np.float32)
        self._check(_lib.lib().cr_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "cr_mlp_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAM
        self._check(_lib.lib().cr_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "cr_mlp_set_params")

    def grads(self) -> np.ndarray:
        g = np.zeros(NPARAM, dtype=np.float32)
        self._check(_lib.lib().cr_mlp_get_grads(self.h, g.ctypes.data_as(C.POINTER(C.c_float))), "cr_mlp_get_grads")
        return g

    def _features(self, x):
        t = self.torch
        if not (isinstance(x, t.Tensor) and x.is_cuda):
            x = t.as_tensor(np.ascontiguousarray(x, dtype=np.uint16).view(np.int16), device="cuda")
        assert x.dtype in (t.int16, t.bfloat16) and x.shape[-1] == FEATURES and x.is_contiguous()
        return x

    def forward(self, x):
        """x: [n, 48] BF16 features (a bfloat16/int16 CUDA tensor or uint16 array) -> y [n] float32."""
        x = self._features(x)
        n = x.shape[0]
        y = self.torch.empty(n, dtype=self.torch.float32, device="cuda")
        self._check(_lib.lib().cr_mlp_forward(self.h, n, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                              self._stream()), "cr_mlp_forward")
        return y

    def accumulate_grad(self, x, target) -> float:
        x = self._features(x)
        t = self.torch
        target = t.as_tensor(target, dtype=t.float32, device="cuda").contiguous()
        loss = C.c_double(0.0)
        self._check(_lib.lib().cr_mlp_accumulate_grad(self.h, x.shape[0], C.c_void_p(x.data_ptr()),
                                                      C.c_void_p(target.data_ptr()), C.byref(loss), self._stream()),
                    "cr_mlp_accumulate_grad")
        return loss.value

    def adam(self, lr=1e-3, clip=1.0):
        self._check(_lib.lib().cr_mlp_adam(self.h, C.c_double(lr), C.c_double(clip), self._stream()), "cr_mlp_adam")

    def train_step(self, x, target, lr=1e-3, clip=1.0) -> float:
        loss = self.accumulate_grad(x, target)
        self.adam(lr, clip)
        return loss

    def set_wait(self, max_cycles: int = 1 << 31, withhold_next: bool = False):
        """Cycle limit of the kernels' bounded barrier waits; withhold_next makes the next
        launch withhold its first MMAs so that its waits run out (timeout-path test hook)."""
        self._check(_lib.lib().cr_mlp_set_wait(self.h, int(max_cycles), int(bool(withhold_next))), "cr_mlp_set_wait")

    def counters(self) -> dict:
        a, b = C.c_longlong(0), C.c_longlong(0)
        self._check(_lib.lib().cr_mlp_counters(self.h, C.byref(a), C.byref(b)), "cr_mlp_counters")
        return {"kernel_launches": a.value, "adam_steps": b.value}
