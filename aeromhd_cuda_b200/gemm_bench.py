"""Timing of the corrector's GEMMs on the three tensor-core paths of the
library: mma.sync (amhd_nn_gemm with path 1: BF16 operands, FP32
accumulation in registers), tcgen05 (amhd_nn_gemm_tc: FP32 accumulator in
tensor memory, operands by TMA where they qualify) and the per-shape choice
amhd_nn_gemm makes by default (path 0), on the shapes a 256x64 U-Net training
step issues (batch 16): forward convolutions (M = output channels, N =
pixels, K = 9 x input channels), the weight gradient (K = pixels, split 8
ways) and the input gradient (A transposed).  --train-step also times one
Adam step of that network (forward, backward, update) on mma.sync only and
with the default choice.

    python -m aeromhd_cuda_b200.gemm_bench [--shapes tA,tB,M,N,K ...] [--iters 20] [--warmup 3] [--train-step]
                                           [--graph]

Prints one JSON object: per shape and path the mean time of a launch (CUDA
events around `iters` back-to-back launches) and its TFLOP/s.  Each launch is
a call from Python through the C ABI (tensor maps encoded on the host per
call), so small shapes can be bound by the host; --graph captures the `iters`
launches into one CUDA graph and times its replay instead (the kernels alone,
as the captured training step runs them).
"""
from __future__ import annotations

import argparse
import ctypes
import json

CORRECTOR_SHAPES = [(0, 0, 32, 262144, 90), (0, 0, 64, 65536, 288), (0, 0, 128, 16384, 576),
                    (0, 0, 256, 4096, 1152), (0, 1, 64, 288, 65536), (1, 0, 288, 65536, 64)]
PATHS = {"mma.sync": ("amhd_nn_gemm", 1), "tcgen05": ("amhd_nn_gemm_tc", 0), "auto": ("amhd_nn_gemm", 0)}


def _events_ms(fn, iters: int, warmup: int, graph: bool = False) -> float:
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if graph:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(iters):
                fn()
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / iters
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / iters


def _check_waits() -> None:
    from . import _lib
    flag = ctypes.c_int32(0)
    _lib.call("amhd_nn_gemm_status", ctypes.byref(flag))
    if flag.value:
        raise RuntimeError("amhd_nn_gemm_tc: a tensor-core wait timed out")


def time_shape(tA: int, tB: int, M: int, N: int, K: int, iters: int, warmup: int, paths=tuple(PATHS),
               graph: bool = False) -> dict:
    import torch
    from . import _lib
    from ._tensors import stream_ptr
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((K, M) if tA else (M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K) if tB else (K, N), device="cuda", generator=g).to(torch.bfloat16)
    C = torch.zeros((M, N), device="cuda")
    splits = 8 if K >= 16384 else 1
    out = {}
    try:
        for name in paths:
            fn_name, mode = PATHS[name]
            _lib.call("amhd_nn_set_gemm_path", mode)

            def launch():
                _lib.call(fn_name, tA, tB, M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1],
                          C.data_ptr(), N, 1.0, 0.0, splits, stream_ptr())
            ms = _events_ms(launch, iters, warmup, graph)
            out[name] = {"ms": round(ms, 4), "TFLOP/s": round(2.0 * M * N * K / ms / 1e9, 2)}
    finally:
        _lib.call("amhd_nn_set_gemm_path", 0)
    _check_waits()
    return out


def time_train_step(iters: int, warmup: int, H: int = 256, W: int = 64, batch: int = 16) -> dict:
    """One Adam step of the corrector U-Net on a batch of random inputs."""
    import torch
    from . import _lib
    from .corrector import Corrector
    net = Corrector(H, W, seed=1)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((10, batch * H * W), device="cuda", generator=g)
    t = torch.randn((10, batch * H * W), device="cuda", generator=g) * 0.1
    out = {}
    try:
        for name, mode in (("mma.sync", 1), ("auto", 0)):
            _lib.call("amhd_nn_set_gemm_path", mode)
            ms = _events_ms(lambda: net.train_step(x, t, batch, lr=1e-5), iters, warmup)
            out[name] = {"ms": round(ms, 3)}
        # the same step replayed as one CUDA graph (library GEMM choice)
        ms = _events_ms(lambda: net.train_step_graphed(x, t, batch, lr=1e-5), iters, warmup)
        out["auto, CUDA graph"] = {"ms": round(ms, 3)}
    finally:
        _lib.call("amhd_nn_set_gemm_path", 0)
    _check_waits()
    return out


def profile_steps(steps: int = 2, H: int = 256, W: int = 64, batch: int = 16) -> None:
    """`steps` eager Adam steps of the corrector U-Net on random inputs with the
    library's GEMM choice and nothing else (a short program for a launch list)."""
    import torch
    from .corrector import Corrector
    net = Corrector(H, W, seed=1)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((10, batch * H * W), device="cuda", generator=g)
    t = torch.randn((10, batch * H * W), device="cuda", generator=g) * 0.1
    for _ in range(steps):
        net.train_step(x, t, batch, lr=1e-5)
        torch.cuda.synchronize()
    _check_waits()


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--shapes", nargs="*", default=None, help="tA,tB,M,N,K (default: the corrector's shapes)")
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--train-step", action="store_true")
    ap.add_argument("--graph", action="store_true", help="time the launches replayed as one CUDA graph")
    ap.add_argument("--profile-step", action="store_true",
                    help="only run two eager training steps (for a profiler's launch list) and print nothing")
    args = ap.parse_args(argv)
    if args.profile_step:
        profile_steps()
        return
    shapes = CORRECTOR_SHAPES if not args.shapes else [tuple(int(x) for x in s.split(",")) for s in args.shapes]
    res = {}
    for (tA, tB, M, N, K) in shapes:
        res[f"{tA}{tB} {M}x{N}x{K}"] = time_shape(tA, tB, M, N, K, args.iters, args.warmup, graph=args.graph)
    if args.train_step:
        res["train_step 256x64 batch 16"] = time_train_step(args.iters, args.warmup)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
