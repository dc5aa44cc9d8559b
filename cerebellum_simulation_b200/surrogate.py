"""Python view of the sweep surrogate (include/cbm_surrogate.h): a small ReLU
MLP trained and evaluated by the library's BF16 tensor-core kernels."""
import ctypes

import numpy as np

from . import lib, _check, CBMError

_P, _U, _U64, _F, _I = ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint64, ctypes.c_float, ctypes.c_int
for _name, (_res, _args) in {
    "cbm_mlp_create": (_I, [_U, _U, _U, _U, _U, _U64, _I, _P]),
    "cbm_mlp_destroy": (None, [_P]),
    "cbm_mlp_num_params": (_U64, [_P]),
    "cbm_mlp_layout": (_I, [_P, _P, _P, _P, _P]),
    "cbm_mlp_get_params": (_I, [_P, _P, _U64]),
    "cbm_mlp_set_params": (_I, [_P, _P, _U64]),
    "cbm_mlp_forward": (_I, [_P, _P, _U, _P]),
    "cbm_mlp_gradients": (_I, [_P, _P, _P, _U, _P, _P]),
    "cbm_mlp_train": (_I, [_P, _P, _P, _U, _U, _U, _F, _U64, _P]),
}.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class MLP:
    """nIn -> h1 -> h2 -> nOut ReLU network on GPU `device`."""

    def __init__(self, n_in, h1, h2, n_out, max_batch=256, seed=0, device=0):
        self.sizes = (n_in, h1, h2, n_out)
        self._h = ctypes.c_void_p()
        _check(lib.cbm_mlp_create(n_in, h1, h2, n_out, max_batch, seed, device, ctypes.byref(self._h)))
        v = [ctypes.c_uint() for _ in range(4)]
        _check(lib.cbm_mlp_layout(self._h, *[ctypes.byref(x) for x in v]))
        self.padded = tuple(x.value for x in v)
        self.max_batch = max_batch

    def __del__(self):
        if getattr(self, "_h", None):
            lib.cbm_mlp_destroy(self._h)
            self._h = None

    def num_params(self):
        return lib.cbm_mlp_num_params(self._h)

    def get_params(self):
        p = np.empty(self.num_params(), dtype=np.float32)
        _check(lib.cbm_mlp_get_params(self._h, p.ctypes.data, p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib.cbm_mlp_set_params(self._h, p.ctypes.data, p.size))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty((x.shape[0], self.sizes[3]), dtype=np.float32)
        _check(lib.cbm_mlp_forward(self._h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib.cbm_mlp_gradients(self._h, x.ctypes.data, t.ctypes.data, x.shape[0], g.ctypes.data,
                                     ctypes.byref(loss)))
        return g, loss.value

    def train(self, x, t, batch=256, epochs=10, lr=1e-3, seed=0):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib.cbm_mlp_train(self._h, x.ctypes.data, t.ctypes.data, x.shape[0], batch, epochs, lr, seed,
                                 ctypes.byref(loss)))
        return loss.value

    def unpack(self, p):
        """(W1, b1, W2, b2, W3, b3) views of a parameter vector, padded shapes."""
        I, H1, H2, O = self.padded
        shapes = [(H1, I), (H1,), (H2, H1), (H2,), (O, H2), (O,)]
        out, k = [], 0
        for s in shapes:
            n = int(np.prod(s))
            out.append(p[k:k + n].reshape(s))
            k += n
        return out
