"""Coordinate MLP of the learned warm start (libpsst_b200's psst_mlp_* and
psst_tc_gemm_bf16 entry points); device buffers are torch CUDA tensors.

Inputs (Mach, ramp angle, x, y) and outputs (rho, u, v, p) are normalised by
the caller; `normalise_inputs` / `targets` / `prim_from_outputs` below give the
convention the warm start uses.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check

MACH_RANGE = (1.8, 4.0)
ANGLE_RANGE = (5.0, 20.0)
X_RANGE = (0.0, 3.0)
Y_RANGE = (0.0, 1.0)


def _scale(v, lo, hi):
    return 2.0 * (np.asarray(v, dtype=np.float64) - lo) / (hi - lo) - 1.0


def normalise_inputs(mach, angle, xy):
    """[n][4] FP32 network inputs for the cells at xy[n][2] of one case."""
    n = len(xy)
    out = np.empty((n, 4), dtype=np.float32)
    out[:, 0] = _scale(mach, *MACH_RANGE)
    out[:, 1] = _scale(angle, *ANGLE_RANGE)
    out[:, 2] = _scale(xy[:, 0], *X_RANGE)
    out[:, 3] = _scale(xy[:, 1], *Y_RANGE)
    return out


def targets(rho, u, v, p, rho_inf, speed_inf, p_inf):
    """[n][4] FP32 targets: fields relative to the freestream, minus 1 for rho and p."""
    return np.stack([rho / rho_inf - 1.0, u / speed_inf, v / speed_inf, p / p_inf - 1.0], axis=1).astype(np.float32)


def fields_from_outputs(y, rho_inf, speed_inf, p_inf):
    """Inverse of `targets`: (rho, u, v, p)."""
    y = np.asarray(y, dtype=np.float64)
    return (y[:, 0] + 1.0) * rho_inf, y[:, 1] * speed_inf, y[:, 2] * speed_inf, (y[:, 3] + 1.0) * p_inf


class MLP:
    """psst_mlp: parameters, Adam state and workspace on one GPU."""

    def __init__(self, device=0, seed=0):
        h = ctypes.c_void_p()
        check(_lib.load().psst_mlp_create(int(device), int(seed), ctypes.byref(h)))
        self._h = h
        self.n = _lib.load().psst_mlp_param_count(self._h)

    def params(self):
        out = np.zeros(self.n, dtype=np.float32)
        check(_lib.load().psst_mlp_get_params(self._h, out.ctypes.data, self.n))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(_lib.load().psst_mlp_set_params(self._h, p.ctypes.data, self.n))

    def _on_torch_stream(self):
        """The network's kernels run on torch's current stream, in order with
        the kernels that made the input tensors and before any that read the
        outputs (the library's own stream would race with both). Torch's
        default stream is the legacy NULL stream (handle 0), which the library
        would take for "its own stream": it is passed as cudaStreamLegacy."""
        import torch

        self.set_stream(torch.cuda.current_stream().cuda_stream or CUDA_STREAM_LEGACY)

    def forward(self, x):
        """x: torch CUDA FP32 [B][4] -> torch CUDA FP32 [B][4]."""
        import torch

        self._on_torch_stream()
        y = torch.empty((x.shape[0], 4), dtype=torch.float32, device=x.device)
        check(_lib.load().psst_mlp_forward(self._h, x.data_ptr(), int(x.shape[0]), y.data_ptr()))
        return y

    def gradients(self, x, t):
        self._on_torch_stream()
        g = np.zeros(self.n, dtype=np.float32)
        loss = ctypes.c_float()
        check(_lib.load().psst_mlp_gradients(self._h, x.data_ptr(), t.data_ptr(), int(x.shape[0]), g.ctypes.data,
                                              ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, x, t, lr):
        self._on_torch_stream()
        loss = ctypes.c_float()
        check(_lib.load().psst_mlp_train_step(self._h, x.data_ptr(), t.data_ptr(), int(x.shape[0]), float(lr),
                                               ctypes.byref(loss)))
        return loss.value

    def set_stream(self, stream_ptr):
        check(_lib.load().psst_mlp_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().psst_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy: the legacy default stream, by its explicit handle


def tc_gemm(A, B, k_split=None, a_strides=None, b_strides=None, M=None, N=None, K=None, wait_polls=None, out=None):
    """D = A . B^T on the tensor cores. A [M][K], B [N][K] torch CUDA BF16 (or
    any strides given explicitly); returns FP32 [splits][M][N] partials.
    wait_polls: bound of the first mbarrier wait (psst_tc_gemm_bf16_wait);
    out: a preallocated [splits][M][N] FP32 result."""
    import torch

    M = M if M is not None else A.shape[0]
    K = K if K is not None else A.shape[1]
    N = N if N is not None else B.shape[0]
    a_sm, a_sk = a_strides if a_strides else A.stride()
    b_sn, b_sk = b_strides if b_strides else B.stride()
    k_split = k_split or max(K, 1)
    splits = max(1, -(-K // k_split))
    D = out if out is not None else torch.zeros((splits, M, N), dtype=torch.float32, device=A.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if wait_polls is None:
        check(_lib.load().psst_tc_gemm_bf16(A.data_ptr(), a_sm, a_sk, B.data_ptr(), b_sn, b_sk, M, N, K, k_split,
                                             D.data_ptr(), N, stream))
    else:
        check(_lib.load().psst_tc_gemm_bf16_wait(A.data_ptr(), a_sm, a_sk, B.data_ptr(), b_sn, b_sk, M, N, K,
                                                  k_split, D.data_ptr(), N, stream, int(wait_polls)))
    return D


def tc_gemm_time(A, B, reps=20, k_split=None, a_strides=None, b_strides=None, M=None, N=None, K=None):
    """Mean device milliseconds of one tensor-core GEMM launch (reps launches
    back to back between CUDA events); same operands as tc_gemm."""
    import torch

    M = M if M is not None else A.shape[0]
    K = K if K is not None else A.shape[1]
    N = N if N is not None else B.shape[0]
    a_sm, a_sk = a_strides if a_strides else A.stride()
    b_sn, b_sk = b_strides if b_strides else B.stride()
    k_split = k_split or max(K, 1)
    splits = max(1, -(-K // k_split))
    D = torch.empty((splits, M, N), dtype=torch.float32, device=A.device)
    ms = ctypes.c_double()
    check(_lib.load().psst_tc_gemm_bf16_time(A.data_ptr(), a_sm, a_sk, B.data_ptr(), b_sn, b_sk, M, N, K, k_split,
                                              D.data_ptr(), N, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                              int(reps), ctypes.byref(ms)))
    return ms.value
