"""Learned per-cycle power proxy (include/gtpb200_proxy.h) from Python.

The network, its training step and its inference run in libgtpb200.so on
the tcgen05 tensor cores; torch tensors here only hold device memory.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi


def _torch():
    import torch
    return torch


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


@dataclass
class ProxyParams:
    W1: np.ndarray
    b1: np.ndarray
    W2: np.ndarray
    b2: np.ndarray
    W3: np.ndarray
    b3: np.ndarray

    def flat(self) -> np.ndarray:
        return np.concatenate([a.reshape(-1) for a in (self.W1, self.b1, self.W2, self.b2, self.W3, self.b3)]
                              ).astype(np.float32)


class PowerProxy:
    """BF16 MLP n_in -> n_hidden -> n_hidden -> n_out on one GPU."""

    def __init__(self, n_in: int = 4096, n_hidden: int = 512, n_out: int = 33, batch: int = 1024,
                 lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
                 weight_decay: float = 0.0, seed: int = 20261203, device: int = 0, use_graph: bool = True):
        self.L = _abi.lib()
        cfg = _abi.gtp_proxy_config()
        self.L.gtp_proxy_config_default(C.byref(cfg))
        cfg.cuda_device_id = device
        cfg.n_in, cfg.n_hidden, cfg.n_out, cfg.batch = n_in, n_hidden, n_out, batch
        cfg.lr, cfg.beta1, cfg.beta2, cfg.eps = lr, beta1, beta2, eps
        cfg.weight_decay = weight_decay
        cfg.seed = seed
        cfg.use_graph = 1 if use_graph else 0
        h = C.c_void_p()
        st = self.L.gtp_proxy_create(C.byref(cfg), C.byref(h))
        if st != _abi.GTP_OK:
            raise _abi.GtpError(st, "gtp_proxy_create failed")
        self.h = h
        self.n_in, self.n_hidden, self.n_out, self.batch = n_in, n_hidden, n_out, batch
        self.device = device
        self._keep = None

    # -- lifecycle --------------------------------------------------------
    def close(self) -> None:
        if self.h:
            self.L.gtp_proxy_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _abi.GTP_OK:
            msg = self.L.gtp_proxy_last_error(self.h)
            raise _abi.GtpError(st, msg.decode() if msg else "")

    @property
    def stream(self):
        """The proxy's CUDA stream as a torch stream object."""
        torch = _torch()
        return torch.cuda.ExternalStream(self.L.gtp_proxy_get_stream(self.h), device=f"cuda:{self.device}")

    @property
    def n_param(self) -> int:
        return int(self.L.gtp_proxy_n_param(self.h))

    # -- training ----------------------------------------------------------
    def set_training_data(self, x, y) -> None:
        """x: [n, n_in] torch.bfloat16 (0/1) on the GPU; y: [n, n_out] float32."""
        torch = _torch()
        assert x.dtype == torch.bfloat16 and x.is_contiguous() and x.shape[1] == self.n_in
        assert y.dtype == torch.float32 and y.is_contiguous() and y.shape == (x.shape[0], self.n_out)
        torch.cuda.current_stream().synchronize()
        self._keep = (x, y)
        self._check(self.L.gtp_proxy_set_training_data(self.h, _ptr(x), _ptr(y), x.shape[0]))

    def norm(self) -> tuple[np.ndarray, np.ndarray]:
        m = np.zeros(self.n_out, np.float32)
        s = np.zeros(self.n_out, np.float32)
        self._check(self.L.gtp_proxy_get_norm(self.h, m.ctypes.data_as(C.c_void_p), s.ctypes.data_as(C.c_void_p)))
        return m, s

    def train(self, epochs: int) -> np.ndarray:
        losses = np.zeros(max(1, epochs), np.float32)
        self._check(self.L.gtp_proxy_train(self.h, epochs, losses.ctypes.data_as(C.c_void_p)))
        return losses[:epochs]

    def compute_grads(self, rows: np.ndarray) -> float:
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        assert rows.shape == (self.batch,)
        loss = C.c_float()
        self._check(self.L.gtp_proxy_compute_grads(self.h, rows.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return float(loss.value)

    def adam_step(self) -> None:
        self._check(self.L.gtp_proxy_adam_step(self.h))

    # -- parameters ----------------------------------------------------------
    def params_flat(self) -> np.ndarray:
        out = np.zeros(self.n_param, np.float32)
        self._check(self.L.gtp_proxy_get_params(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def grads_flat(self) -> np.ndarray:
        out = np.zeros(self.n_param, np.float32)
        self._check(self.L.gtp_proxy_get_grads(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params_flat(self, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float32)
        assert v.shape == (self.n_param,)
        self._check(self.L.gtp_proxy_set_params(self.h, v.ctypes.data_as(C.c_void_p)))

    def unflatten(self, v: np.ndarray) -> ProxyParams:
        I, H, O = self.n_in, self.n_hidden, self.n_out
        sizes = [H * I, H, H * H, H, O * H, O]
        parts = np.split(np.asarray(v), np.cumsum(sizes)[:-1])
        return ProxyParams(parts[0].reshape(H, I), parts[1], parts[2].reshape(H, H), parts[3],
                           parts[4].reshape(O, H), parts[5])

    # -- inference -----------------------------------------------------------
    def predict(self, x, out=None, sync: bool = True):
        """x: [n, n_in] torch.bfloat16 on the GPU -> [n, n_out] float32."""
        torch = _torch()
        assert x.dtype == torch.bfloat16 and x.is_contiguous() and x.shape[1] == self.n_in
        n = x.shape[0]
        if out is None:
            out = torch.empty((n, self.n_out), dtype=torch.float32, device=x.device)
        # x and out come from torch's current stream: the proxy's stream waits
        # for it on the device, with no host stall
        self.stream.wait_stream(torch.cuda.current_stream())
        self._check(self.L.gtp_proxy_predict(self.h, _ptr(x), n, _ptr(out)))
        if sync:
            self.stream.synchronize()
        return out


def toggle_bits(net_off, time, sel, ticks_per_cycle: int, c_lo: int, c_hi: int, out=None, stream=None):
    """[c_hi - c_lo, len(sel)] BF16 toggle bits of the selected nets from a
    device event CSR (net_off int64 [n_net+1], time int64 [n_event])."""
    torch = _torch()
    L = _abi.lib()
    n_sel = int(sel.shape[0])
    if out is None:
        out = torch.zeros((c_hi - c_lo, n_sel), dtype=torch.bfloat16, device=net_off.device)
    st = L.gtp_toggle_bits(_ptr(net_off), _ptr(time), _ptr(sel), n_sel, ticks_per_cycle, c_lo, c_hi,
                           _ptr(out), out.stride(0), C.c_void_p(stream or 0))
    _abi.check(st)
    return out


def toggle_bits_windows(windows, sel, ticks_per_cycle: int, c_base: int, out, stream=None) -> None:
    """Dense toggle bits of several windows: windows is a list of (net_off,
    time, c_lo, c_hi) with device event CSRs and disjoint cycle ranges;
    out[c - c_base, k] = 1.0 or 0.0 for every c in a window's range and
    k < len(sel). Rows outside the windows are left as they are."""
    L = _abi.lib()
    n_sel = int(sel.shape[0])
    for i in range(0, len(windows), _abi.BITS_MAX_WINDOWS):
        part = windows[i:i + _abi.BITS_MAX_WINDOWS]
        arr = (_abi.gtp_bits_window * len(part))(*[
            _abi.gtp_bits_window(_ptr(no), _ptr(tm), int(lo), int(hi)) for no, tm, lo, hi in part])
        _abi.check(L.gtp_toggle_bits_windows(arr, len(part), _ptr(sel), n_sel, ticks_per_cycle, c_base,
                                             _ptr(out), out.stride(0), C.c_void_p(stream or 0)))


def net_toggle_stats(net_off, time, n_net: int, ticks_per_cycle: int, c_lo: int, c_hi: int, y,
                     count=None, sum_y=None, stream=None):
    """Per net: number of toggling cycles in [c_lo, c_hi) and the sum of
    y[c - c_lo] over them (accumulated into count / sum_y when given)."""
    torch = _torch()
    L = _abi.lib()
    dev = net_off.device
    if count is None:
        count = torch.zeros(n_net, dtype=torch.int64, device=dev)
    if sum_y is None:
        sum_y = torch.zeros(n_net, dtype=torch.float64, device=dev)
    st = L.gtp_net_toggle_stats(_ptr(net_off), _ptr(time), n_net, ticks_per_cycle, c_lo, c_hi, _ptr(y),
                                _ptr(count), _ptr(sum_y), C.c_void_p(stream or 0))
    _abi.check(st)
    return count, sum_y


def bf16_gemm(a, b, bias=None, relu: bool = False, stream=None):
    """a [m, k] bf16, b [n, k] bf16 -> a @ b.T (+ bias, relu) in float32, on
    the tcgen05 GEMM."""
    torch = _torch()
    L = _abi.lib()
    m, k = a.shape
    n = b.shape[0]
    c = torch.empty((m, n), dtype=torch.float32, device=a.device)
    st = L.gtp_bf16_gemm(_ptr(a), a.stride(0), _ptr(b), b.stride(0), m, n, k,
                         _ptr(bias) if bias is not None else None, 1 if relu else 0, _ptr(c), n,
                         C.c_void_p(stream or 0))
    _abi.check(st)
    return c
