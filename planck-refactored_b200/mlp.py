"""ctypes binding of the learned-guess network (pfk_mlp_* in the C ABI).

The network's forward pass, gradients and Adam updates run in the library's
BF16 tensor-core kernels (csrc/pfk_mlp.cu); this module only owns the handle,
moves parameters, and passes device pointers of torch tensors (device memory
and streams are the only things torch provides here)."""
import ctypes

import numpy as np

from . import PFK_OK, PfkError, load_library


def _bind(L):
    if getattr(L, "_pfk_mlp_bound", False):
        return L
    vp, c_int, c_ll, c_f, c_d = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    for n in ("pfk_mlp_create", "pfk_mlp_destroy", "pfk_mlp_set_params", "pfk_mlp_get_params", "pfk_mlp_forward",
              "pfk_mlp_gradients", "pfk_mlp_train_step"):
        getattr(L, n).restype = c_int
    L.pfk_mlp_create.argtypes = [c_int, vp, c_int, c_int, ctypes.POINTER(vp)]
    L.pfk_mlp_destroy.argtypes = [vp]
    L.pfk_mlp_last_error.restype = ctypes.c_char_p
    L.pfk_mlp_last_error.argtypes = [vp]
    L.pfk_mlp_param_count.restype = c_ll
    L.pfk_mlp_param_count.argtypes = [vp]
    L.pfk_mlp_set_params.argtypes = [vp, vp]
    L.pfk_mlp_get_params.argtypes = [vp, vp]
    L.pfk_mlp_forward.argtypes = [vp, vp, c_int, vp, vp]
    L.pfk_mlp_gradients.argtypes = [vp, vp, vp, c_int, vp, ctypes.POINTER(c_d), vp]
    L.pfk_mlp_train_step.argtypes = [vp, vp, vp, c_int, c_f, ctypes.POINTER(c_d), vp]
    L._pfk_mlp_bound = True
    return L


def init_params(dims, seed=0):
    """Uniform(+-sqrt(6 / fan_in)) weights (He-style for SiLU), zero biases."""
    rng = np.random.default_rng(seed)
    out = []
    for din, dout in zip(dims[:-1], dims[1:]):
        lim = np.sqrt(6.0 / din)
        out.append(rng.uniform(-lim, lim, (din, dout)).astype(np.float32).ravel())
        out.append(np.zeros(dout, dtype=np.float32))
    return np.concatenate(out)


class MLP:
    """dims[0] -> ... -> dims[-1] network on one GPU (widths multiples of 8)."""

    def __init__(self, dims, max_batch, device=0, seed=0, params=None):
        self.L = _bind(load_library())
        self.dims = [int(d) for d in dims]
        self.max_batch, self.device = int(max_batch), int(device)
        d = (ctypes.c_int * len(self.dims))(*self.dims)
        h = ctypes.c_void_p()
        st = self.L.pfk_mlp_create(len(self.dims) - 1, ctypes.cast(d, ctypes.c_void_p), self.max_batch,
                                   self.device, ctypes.byref(h))
        if st != PFK_OK:
            raise PfkError(st, self.L.pfk_mlp_last_error(None).decode())
        self.h = h
        self.nparam = int(self.L.pfk_mlp_param_count(h))
        self.set_params(init_params(self.dims, seed) if params is None else params)

    def _check(self, st):
        if st != PFK_OK:
            raise PfkError(st, self.L.pfk_mlp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.pfk_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparam
        self._check(self.L.pfk_mlp_set_params(self.h, p.ctypes.data))

    def params(self):
        p = np.zeros(self.nparam, dtype=np.float32)
        self._check(self.L.pfk_mlp_get_params(self.h, p.ctypes.data))
        return p

    @staticmethod
    def _ptr(t):
        assert t.is_cuda and t.dtype.is_floating_point and t.is_contiguous()
        return ctypes.c_void_p(t.data_ptr())

    def forward(self, X, stream=None):
        """X: contiguous float32 CUDA tensor (n x dims[0]); returns (n x dims[-1])."""
        import torch
        Y = torch.empty((X.shape[0], self.dims[-1]), device=X.device, dtype=torch.float32)
        st = stream.cuda_stream if stream is not None else None
        self._check(self.L.pfk_mlp_forward(self.h, self._ptr(X), int(X.shape[0]), self._ptr(Y), st))
        return Y

    def gradients(self, X, T, stream=None):
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = ctypes.c_double()
        st = stream.cuda_stream if stream is not None else None
        self._check(self.L.pfk_mlp_gradients(self.h, self._ptr(X), self._ptr(T), int(X.shape[0]), g.ctypes.data,
                                             ctypes.byref(loss), st))
        return g, loss.value

    def train_step(self, X, T, lr, stream=None):
        loss = ctypes.c_double()
        st = stream.cuda_stream if stream is not None else None
        self._check(self.L.pfk_mlp_train_step(self.h, self._ptr(X), self._ptr(T), int(X.shape[0]), float(lr),
                                              ctypes.byref(loss), st))
        return loss.value

    def unpack(self, p=None):
        """[(W_l, b_l)] from a parameter vector (the C ABI's layout)."""
        p = self.params() if p is None else p
        out, o = [], 0
        for din, dout in zip(self.dims[:-1], self.dims[1:]):
            W = p[o:o + din * dout].reshape(din, dout)
            o += din * dout
            b = p[o:o + dout]
            o += dout
            out.append((W, b))
        return out
