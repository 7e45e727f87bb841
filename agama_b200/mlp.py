"""The bracket-predictor network on the device (6 -> 128 -> 128 -> 128 -> 3, SiLU; tcgen05 BF16
hidden products with FP32 accumulation, FP32 master parameters, Adam).

    net = BracketNet(seed)
    history = net.train(x, t, mask, epochs=..., batch=..., lr=...)   # raw inputs / targets
    y = net.predict(x)                                               # numpy or CUDA tensor
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, ptr, F


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class BracketNet:
    def __init__(self, seed=0):
        h = _native.lib().agama_mlpCreate(int(seed))
        if not h:
            raise RuntimeError("agama_b200: " + _native.error())
        self._h = ctypes.c_void_p(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_native, "_lib", None)     # module globals may be gone at interpreter exit
        if h and lib is not None:
            lib.agama_mlpDelete(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @staticmethod
    def num_params():
        return _native.lib().agama_mlpNumParams()

    def params(self):
        """(flat FP32 parameters, scaling[18])"""
        p, s = np.empty(self.num_params(), dtype=np.float32), np.empty(18, dtype=np.float32)
        check(_native.lib().agama_mlpGetParams(self._h, ptr(p, F), ptr(s, F)))
        return p, s

    def set_params(self, params=None, scaling=None):
        p = None if params is None else _f32(params)
        s = None if scaling is None else _f32(scaling)
        check(_native.lib().agama_mlpSetParams(self._h, ptr(p, F), ptr(s, F)))

    def loss_grad(self, x, t, mask):
        """loss and gradient of one batch of standardised inputs / targets (batch % 128 == 0)"""
        x, t, m = _f32(x), _f32(t), _f32(mask)
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = ctypes.c_float(0)
        check(_native.lib().agama_mlpLossGrad(self._h, len(x), ptr(x, F), ptr(t, F), ptr(m, F), ptr(g, F),
                                              ctypes.byref(loss)))
        return loss.value, g

    def train(self, x, t, mask, epochs=10, batch=1024, lr=2e-3, seed=0):
        """Adam on raw samples (the input / output standardisation is derived from them);
        returns the mean loss of each epoch (standardised units)"""
        x, t, m = _f32(x), _f32(t), _f32(mask)
        hist = np.empty(epochs, dtype=np.float32)
        check(_native.lib().agama_mlpTrain(self._h, len(x), ptr(x, F), ptr(t, F), ptr(m, F), int(epochs), int(batch),
                                           float(lr), int(seed), ptr(hist, F)))
        return hist

    def predict(self, x):
        """predictions (n x 3) for raw inputs (n x 6): numpy in -> numpy out, CUDA tensor in -> tensor out"""
        import torch
        from . import _is_device_array, _current_stream
        dev = _is_device_array(x)
        xd = x.contiguous().float() if dev else torch.tensor(_f32(x), device="cuda")
        y = torch.empty((xd.shape[0], 3), dtype=torch.float32, device=xd.device)
        check(_native.lib().agama_mlpPredictDevice(self._h, xd.shape[0], ctypes.c_void_p(xd.data_ptr()),
                                                   ctypes.c_void_p(y.data_ptr()), _current_stream()))
        if dev:
            return y
        out = y.cpu().numpy()
        check(_native.lib().agama_mlpCheck(self._h))
        return out
