"""BF16 tensor-core MLP: binding of the ``hexmlp_*`` kernels (include/hexmlp.h)
and a small multilayer perceptron trained and evaluated with them.

All arithmetic of the network (GEMMs with fused bias/GELU epilogues, their
backward products, the loss gradient, bias gradients and Adam) runs in the
library's CUDA kernels; torch tensors only hold device memory.

Layer shapes are padded for the tensor-core tiles: feature and hidden
widths to multiples of 128 (the GEMM's N tile) and the batch to a multiple
of 128 rows; padded inputs are zero and padded outputs are ignored by the
loss, so the padding never changes the valid outputs.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

EPI_F32, EPI_GELU, EPI_GELU_GRAD = 0, 1, 2
TILE_M, TILE_K = 128, 64


class HexMlpGemm(C.Structure):
    _fields_ = [("A", C.c_void_p), ("B", C.c_void_p), ("M", C.c_int32), ("N", C.c_int32), ("K", C.c_int32),
                ("bn", C.c_int32), ("epilogue", C.c_int32), ("bias", C.c_void_p), ("C", C.c_void_p),
                ("Ct", C.c_void_p), ("Z", C.c_void_p), ("Zin", C.c_void_p), ("Cf", C.c_void_p),
                ("err", C.c_void_p), ("kernel", C.c_int32)]


GEMM_PERSISTENT, GEMM_STAGED = 0, 1


MLP_EXPORTS = {
    "hexmlp_gemm": (C.c_int, [C.POINTER(HexMlpGemm), C.c_void_p]),
    "hexmlp_gemm_wait_limit": (C.c_int, [C.POINTER(HexMlpGemm), C.c_uint32, C.c_void_p]),
    "hexmlp_gemm_smem_bytes": (C.c_size_t, [C.c_int]),
    "hexmlp_gemm_tile_rows": (C.c_int, []),
    "hexmlp_gemm_tile_k": (C.c_int, []),
    "hexmlp_mse_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hexmlp_bias_grad": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "hexmlp_pack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "hexmlp_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                              C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, C.c_void_p, C.c_void_p,
                              C.c_void_p]),
}


def load() -> C.CDLL:
    lib = _lib.load()
    if not getattr(lib, "_hexmlp_bound", False):
        for name, (res, args) in MLP_EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        lib._hexmlp_bound = True
    return lib


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc}")


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


def gemm(A, B, *, epilogue: int = EPI_F32, bias=None, C_out=None, Ct=None, Z=None, Zin=None, Cf=None, err=None,
         bn: int | None = None, kernel: int = GEMM_PERSISTENT, mma_wait_polls: int | None = None):
    """C = A . B^T on the tensor cores (see include/hexmlp.h).  ``bn``: the
    output tile width, 128 or 256 (default: 256 where N allows it for the
    persistent kernel, 128 for the staged one).  ``mma_wait_polls`` bounds
    the MMA issuer's wait for each loaded stage (``hexmlp_gemm_wait_limit``,
    a check of the kernel's give-up path; None: the normal limit)."""
    import torch

    M, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K and A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16
    assert A.is_contiguous() and B.is_contiguous()
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=A.device)
    if bn is None:
        bn = 256 if (kernel == GEMM_PERSISTENT and N % 256 == 0) else 128
    p = HexMlpGemm(_ptr(A), _ptr(B), M, N, K, bn, epilogue, _ptr(bias), _ptr(C_out), _ptr(Ct), _ptr(Z), _ptr(Zin),
                   _ptr(Cf), _ptr(err), kernel)
    if mma_wait_polls is None:
        _check(load().hexmlp_gemm(C.byref(p), _stream()), f"hexmlp_gemm {M}x{N}x{K}")
    else:
        _check(load().hexmlp_gemm_wait_limit(C.byref(p), int(mma_wait_polls), _stream()),
               f"hexmlp_gemm_wait_limit {M}x{N}x{K}")
    return err


@dataclass
class Layer:
    """FP32 master weights, Adam moments, and the bf16 copies the GEMMs read."""

    w: object   # float [out][in]
    b: object   # float [out]
    wb: object  # bf16 [out][in]
    wbt: object  # bf16 [in][out]
    m1: object
    m2: object
    bm1: object
    bm2: object
    gw: object  # float [out][in]
    gb: object  # float [out]


class TensorCoreMLP:
    """``n_in -> hidden x depth (GELU) -> n_out`` with bf16 weights and
    activations, FP32 accumulation, trained with Adam on a mean-squared
    error."""

    def __init__(self, n_in: int, hidden: int, depth: int, n_out: int, *, seed: int = 0, device: str = "cuda"):
        import torch

        self.n_in, self.hidden, self.depth, self.n_out = n_in, hidden, depth, n_out
        self.p_in, self.p_hidden, self.p_out = round_up(n_in, 128), round_up(hidden, 128), round_up(n_out, 128)
        dims = [self.p_in] + [self.p_hidden] * depth + [self.p_out]
        real = [n_in] + [hidden] * depth + [n_out]
        gen = np.random.default_rng(seed)
        self.layers: list[Layer] = []
        for i in range(depth + 1):
            fan_in, fan_out = real[i], real[i + 1]
            w = np.zeros((dims[i + 1], dims[i]), dtype=np.float32)
            # He initialisation on the real block; padding rows/columns stay 0
            w[:fan_out, :fan_in] = gen.standard_normal((fan_out, fan_in)) * np.sqrt(2.0 / fan_in)
            if i == depth:
                w[:fan_out, :fan_in] *= 0.1
            wt = torch.from_numpy(w).to(device)
            lay = Layer(w=wt, b=torch.zeros(dims[i + 1], device=device),
                        wb=wt.to(torch.bfloat16).contiguous(), wbt=wt.t().contiguous().to(torch.bfloat16),
                        m1=torch.zeros_like(wt), m2=torch.zeros_like(wt),
                        bm1=torch.zeros(dims[i + 1], device=device), bm2=torch.zeros(dims[i + 1], device=device),
                        gw=torch.zeros_like(wt), gb=torch.zeros(dims[i + 1], device=device))
            self.layers.append(lay)
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self._ws: dict[int, dict] = {}

    # --------------------------------------------------------- workspace
    def _workspace(self, M: int) -> dict:
        import torch

        ws = self._ws.get(M)
        if ws is None:
            dev = self.layers[0].w.device
            bf = dict(dtype=torch.bfloat16, device=dev)
            ws = {"H": [], "Ht": [], "Z": []}
            for _ in range(self.depth):
                ws["H"].append(torch.empty(M, self.p_hidden, **bf))
                ws["Ht"].append(torch.empty(self.p_hidden, M, **bf))
                ws["Z"].append(torch.empty(M, self.p_hidden, **bf))
            ws["Y"] = torch.empty(M, self.p_out, dtype=torch.float32, device=dev)
            ws["dY"] = torch.empty(M, self.p_out, **bf)
            ws["dYt"] = torch.empty(self.p_out, M, **bf)
            ws["dZ"] = torch.empty(M, self.p_hidden, **bf)
            ws["dZt"] = torch.empty(self.p_hidden, M, **bf)
            ws["dZ2"] = torch.empty(M, self.p_hidden, **bf)
            ws["dZt2"] = torch.empty(self.p_hidden, M, **bf)
            ws["Xt"] = torch.empty(self.p_in, M, **bf)
            ws["loss"] = torch.zeros(1, dtype=torch.float32, device=dev)
            self._ws[M] = ws
        return ws

    # ----------------------------------------------------------- forward
    def forward(self, X, *, keep: bool = False):
        """X: bf16 [M][p_in] (M a multiple of 128) -> float [M][p_out]."""
        M = X.shape[0]
        ws = self._workspace(M)
        a = X
        for i in range(self.depth):
            lay = self.layers[i]
            # the pre-activations and transposed activations are kept for the backward pass only
            gemm(a, lay.wb, epilogue=EPI_GELU, bias=lay.b, C_out=ws["H"][i], Ct=ws["Ht"][i] if keep else None,
                 Z=ws["Z"][i] if keep else None, err=self.err)
            a = ws["H"][i]
        last = self.layers[-1]
        gemm(a, last.wb, epilogue=EPI_F32, bias=last.b, Cf=ws["Y"], err=self.err)
        return ws["Y"]

    # ---------------------------------------------------------- training
    def gradients(self, X, Xt, T, m_valid: int):
        """Loss and gradients of the mean squared error over the valid rows
        and outputs; X bf16 [M][p_in], Xt its transpose, T float [M][p_out]."""
        lib = load()
        M = X.shape[0]
        ws = self._workspace(M)
        Y = self.forward(X, keep=True)
        ws["loss"].zero_()
        scale = 1.0 / float(m_valid * self.n_out)
        _check(lib.hexmlp_mse_grad(_ptr(Y), _ptr(T), M, self.p_out, m_valid, self.n_out, scale, _ptr(ws["dY"]),
                                   _ptr(ws["dYt"]), _ptr(ws["loss"]), _stream()), "mse_grad")
        d, dt = ws["dY"], ws["dYt"]
        bufs = [(ws["dZ"], ws["dZt"]), (ws["dZ2"], ws["dZt2"])]
        for i in range(self.depth, -1, -1):
            lay = self.layers[i]
            prev_t = ws["Ht"][i - 1] if i > 0 else Xt
            # dW = dZ^T . A_prev (A_prev^T rows are the B operand), db = sum dZ
            gemm(dt, prev_t, epilogue=EPI_F32, Cf=lay.gw, err=self.err)
            _check(lib.hexmlp_bias_grad(_ptr(dt), dt.shape[0], M, _ptr(lay.gb), _stream()), "bias_grad")
            if i > 0:
                nd, ndt = bufs[i % 2]
                # dA_prev = dZ . W, times GELU'(Z_prev)
                gemm(d, lay.wbt, epilogue=EPI_GELU_GRAD, C_out=nd, Ct=ndt, Zin=ws["Z"][i - 1], err=self.err)
                d, dt = nd, ndt
        return ws["loss"]

    def adam(self, lr: float, *, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, decay: float = 0.0):
        lib = load()
        self.step_count += 1
        st = _stream()
        for lay in self.layers:
            rows, cols = lay.w.shape
            _check(lib.hexmlp_adam(_ptr(lay.w), _ptr(lay.m1), _ptr(lay.m2), _ptr(lay.gw), rows, cols, lr, b1, b2,
                                   eps, self.step_count, decay, _ptr(lay.wb), _ptr(lay.wbt), st), "adam")
            _check(lib.hexmlp_adam(_ptr(lay.b), _ptr(lay.bm1), _ptr(lay.bm2), _ptr(lay.gb), 1, rows, lr, b1, b2,
                                   eps, self.step_count, 0.0, None, None, st), "adam bias")

    def check(self) -> None:
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core GEMM gave up waiting on its MMAs")


def forward_flops(net: TensorCoreMLP, M: int) -> float:
    """FLOPs of one forward pass over M rows at the padded layer widths."""
    dims = [net.p_in] + [net.p_hidden] * net.depth + [net.p_out]
    return 2.0 * M * sum(a * b for a, b in zip(dims[:-1], dims[1:]))


def bench_forward(n_in: int = 330, hidden: int = 512, depth: int = 3, n_out: int = 165, rows: int = 40962,
                  reps: int = 20) -> dict:
    """Time the forward pass of a network over ``rows`` rows (the column
    network over every column of the 40962-cell mesh by default) with CUDA
    events; returns milliseconds and TFLOP/s at the padded widths."""
    import torch

    net = TensorCoreMLP(n_in, hidden, depth, n_out, seed=0)
    M = round_up(rows, TILE_M)
    gen = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn(M, net.p_in, device="cuda", generator=gen).to(torch.bfloat16)
    for _ in range(3):
        net.forward(X)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(X)
    e1.record()
    torch.cuda.synchronize()
    net.check()
    ms = e0.elapsed_time(e1) / reps
    flops = forward_flops(net, M)
    return {"rows": M, "shape": f"{net.p_in} -> {net.p_hidden} x{depth} -> {net.p_out}", "ms": ms,
            "tflops": flops / (ms / 1000.0) / 1e12, "gemm_launches": depth + 1}


if __name__ == "__main__":
    import json
    import sys

    if len(sys.argv) > 1 and sys.argv[1] == "--bench":
        print(json.dumps({"column": bench_forward(), "edge": bench_forward(220, 256, 3, 55, rows=122880)}))
