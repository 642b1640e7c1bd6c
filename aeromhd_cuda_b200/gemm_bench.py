"""Timing of the corrector's GEMMs: amhd_nn_gemm (mma.sync, BF16 operands,
FP32 accumulation in registers) against amhd_nn_gemm_tc (tcgen05.mma, FP32
accumulator in tensor memory) on the shapes a 256x64 U-Net training step
issues (batch 16): forward convolutions (M = output channels, N = pixels,
K = 9 x input channels), the weight gradient (K = pixels, split 8 ways) and
the input gradient (A transposed).

    python -m aeromhd_cuda_b200.gemm_bench [--shapes tA,tB,M,N,K ...] [--iters 20] [--warmup 3]

Prints one JSON object: per shape and kernel the mean time of a launch
(CUDA events around `iters` back-to-back launches) and its TFLOP/s.
"""
from __future__ import annotations

import argparse
import json

CORRECTOR_SHAPES = [(0, 0, 32, 262144, 90), (0, 0, 64, 65536, 288), (0, 0, 128, 16384, 576),
                    (0, 0, 256, 4096, 1152), (0, 1, 64, 288, 65536), (1, 0, 288, 65536, 64)]
KERNELS = ("amhd_nn_gemm", "amhd_nn_gemm_tc")


def time_shape(tA: int, tB: int, M: int, N: int, K: int, iters: int, warmup: int, kernels=KERNELS) -> dict:
    import torch
    from . import _lib
    from ._tensors import stream_ptr
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((K, M) if tA else (M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K) if tB else (K, N), device="cuda", generator=g).to(torch.bfloat16)
    C = torch.zeros((M, N), device="cuda")
    splits = 8 if K >= 16384 else 1
    out = {}
    for name in kernels:
        def launch():
            _lib.call(name, tA, tB, M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1], C.data_ptr(), N,
                      1.0, 0.0, splits, stream_ptr())
        for _ in range(warmup):
            launch()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            launch()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / iters
        out[name] = {"ms": round(ms, 4), "TFLOP/s": round(2.0 * M * N * K / ms / 1e9, 2)}
    if "amhd_nn_gemm_tc" in kernels:
        import ctypes
        flag = ctypes.c_int32(0)
        _lib.call("amhd_nn_gemm_status", ctypes.byref(flag))
        if flag.value:
            raise RuntimeError("amhd_nn_gemm_tc: a tensor-core wait timed out")
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--shapes", nargs="*", default=None, help="tA,tB,M,N,K (default: the corrector's shapes)")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    shapes = CORRECTOR_SHAPES if not args.shapes else [tuple(int(x) for x in s.split(",")) for s in args.shapes]
    res = {}
    for (tA, tB, M, N, K) in shapes:
        res[f"{tA}{tB} {M}x{N}x{K}"] = time_shape(tA, tB, M, N, K, args.iters, args.warmup)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
