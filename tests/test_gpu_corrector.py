"""Corrector kernels on the GPU against float32 references: the BF16 GEMM in
every transpose/split variant against a float matmul of the same BF16-rounded
operands; the full network's output and every parameter gradient against the
CPU autograd oracle (tests/nn_oracle.py); Adam against torch.optim.Adam; and
the solver <-> network data movement."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def bf(t):
    return t.to(torch.bfloat16)


@pytest.mark.parametrize("path", [1, 0])
@pytest.mark.parametrize("transA,transB", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,splits", [(37, 91, 53, 1), (128, 300, 700, 4), (10, 4096, 288, 1), (64, 64, 5000, 7),
                                          (256, 320, 704, 4), (32, 2048, 96, 1), (10, 640, 96, 1)])
def test_gemm_matches_float_matmul(transA, transB, M, N, K, splits, path):
    """amhd_nn_gemm on mma.sync (path 1) and with the per-shape choice of
    kernel (path 0: tcgen05 wherever N >= 64 or K >= 4096 and the operands
    qualify, M below a tile included)."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    g = torch.Generator(device="cuda").manual_seed(M * N + K)
    A = bf(torch.randn((K, M) if transA else (M, K), device="cuda", generator=g))
    B = bf(torch.randn((N, K) if transB else (K, N), device="cuda", generator=g))
    C = torch.randn((M, N), device="cuda", generator=g)
    C0 = C.clone()
    _lib.call("amhd_nn_set_gemm_path", path)
    try:
        _lib.call("amhd_nn_gemm", transA, transB, M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1],
                  C.data_ptr(), N, 0.5, 2.0, splits, stream_ptr())
    finally:
        _lib.call("amhd_nn_set_gemm_path", 0)
    opA = A.float().t() if transA else A.float()
    opB = B.float().t() if transB else B.float()
    ref = 0.5 * (opA.double() @ opB.double()) + 2.0 * C0.double()
    err = float((C.double() - ref).abs().max() / ref.abs().max())
    assert err < 2e-6, err


@pytest.mark.parametrize("transA,transB", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (37, 91, 53, 1), (256, 300, 700, 4), (10, 4096, 288, 1),
                                          (64, 64, 5000, 7), (256, 320, 704, 4), (200, 136, 96, 1),
                                          (256, 19200, 200, 1), (130, 12800, 72, 1)])
def test_tcgen05_gemm_matches_float_matmul(transA, transB, M, N, K, splits):
    """amhd_nn_gemm_tc (tcgen05.mma, FP32 accumulator in tensor memory) against a
    float64 matmul of the same BF16 operands, every transpose and split-K case,
    partial tiles included, on both operand paths (TMA pipeline where ld and K
    are multiples of 8, thread staging where not); its waits never gave up."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    import ctypes
    g = torch.Generator(device="cuda").manual_seed(M * N + K + 7)
    A = bf(torch.randn((K, M) if transA else (M, K), device="cuda", generator=g))
    B = bf(torch.randn((N, K) if transB else (K, N), device="cuda", generator=g))
    C = torch.randn((M, N), device="cuda", generator=g)
    C0 = C.clone()
    _lib.call("amhd_nn_gemm_tc", transA, transB, M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1],
              C.data_ptr(), N, 0.5, 2.0, splits, stream_ptr())
    torch.cuda.synchronize()
    flag = ctypes.c_int32(-1)
    _lib.call("amhd_nn_gemm_status", ctypes.byref(flag))
    assert flag.value == 0
    opA = A.float().t() if transA else A.float()
    opB = B.float().t() if transB else B.float()
    ref = 0.5 * (opA.double() @ opB.double()) + 2.0 * C0.double()
    err = float((C.double() - ref).abs().max() / ref.abs().max())
    assert err < 2e-6, err


@pytest.mark.parametrize("transA,transB", [(0, 0), (1, 1), (0, 1)])
@pytest.mark.parametrize("M,N,K", [(256, 19200, 200), (32, 262144, 96), (128, 16384, 576)])
def test_persistent_gemm_equals_one_tile_per_cta(transA, transB, M, N, K):
    """The persistent TMA GEMM (one CTA per SM, several tiles each, two TMEM
    accumulators) and the one-tile-per-CTA kernel accumulate every tile in the
    same K order: identical bits; no wait gave up."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    import ctypes
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = bf(torch.randn((K, M) if transA else (M, K), device="cuda", generator=g))
    B = bf(torch.randn((N, K) if transB else (K, N), device="cuda", generator=g))
    out = []
    try:
        for persistent in (1, 0):
            _lib.call("amhd_nn_set_gemm_persistent", persistent)
            C = torch.full((M, N), float("nan"), device="cuda")
            _lib.call("amhd_nn_gemm_tc", transA, transB, M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1],
                      C.data_ptr(), N, 1.0, 0.0, 1, stream_ptr())
            out.append(C)
    finally:
        _lib.call("amhd_nn_set_gemm_persistent", 1)
    torch.cuda.synchronize()
    flag = ctypes.c_int32(-1)
    _lib.call("amhd_nn_gemm_status", ctypes.byref(flag))
    assert flag.value == 0
    assert torch.isfinite(out[0]).all()
    assert torch.equal(out[0], out[1])


def test_tcgen05_gemm_operand_paths():
    """Operands whose leading dimension is a multiple of 8 go through the TMA
    pipeline (also with a K that is not: the ragged K step reads zeros past
    K), others through thread staging; all agree with the float64 matmul."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    import ctypes

    def paths():
        t, s = ctypes.c_int64(-1), ctypes.c_int64(-1)
        _lib.call("amhd_nn_gemm_tc_paths", ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    for (M, N, K, lda), expect in (((128, 256, 128, 128), (1, 0)), ((128, 256, 90, 90), (0, 1)),
                                   ((136, 200, 100, 104), (1, 0))):
        g = torch.Generator(device="cuda").manual_seed(K)
        A = bf(torch.randn((M, lda), device="cuda", generator=g))[:, :K]
        B = bf(torch.randn((K, N), device="cuda", generator=g))
        C = torch.zeros((M, N), device="cuda")
        t0, s0 = paths()
        _lib.call("amhd_nn_gemm_tc", 0, 0, M, N, K, A.data_ptr(), lda, B.data_ptr(), N, C.data_ptr(), N, 1.0, 0.0, 1,
                  stream_ptr())
        torch.cuda.synchronize()
        t1, s1 = paths()
        assert (t1 - t0, s1 - s0) == expect, (M, N, K, t1 - t0, s1 - s0)
        ref = A.double() @ B.double()
        assert float((C.double() - ref).abs().max() / ref.abs().max()) < 2e-6


def _net_and_oracle(H=32, W=16, B=2, seed=5):
    import nn_oracle
    from aeromhd_cuda_b200.corrector import Corrector, architecture, init_params
    p = init_params(architecture(), seed)
    # make the last layer non-trivial so that gradients are well conditioned
    p["out"]["w"] *= 10.0
    for v in p.values():
        v["b"].normal_(0, 0.05, generator=torch.Generator().manual_seed(seed + 1))
    # round weights to bf16 so both sides use identical operand values
    for v in p.values():
        v["w"] = v["w"].to(torch.bfloat16).float()
    net = Corrector(H, W, params=p)
    gen = torch.Generator().manual_seed(seed + 2)
    x = torch.randn(B, 10, H, W, generator=gen).to(torch.bfloat16).float()
    tgt = torch.randn(B, 10, H, W, generator=gen)
    return net, p, x, tgt, nn_oracle


def test_network_forward_and_gradients_match_cpu_oracle():
    net, p, x, tgt, O = _net_and_oracle()
    B, H, W = x.shape[0], x.shape[2], x.shape[3]
    # oracle
    leaf = {k: {"w": v["w"].clone().requires_grad_(True), "b": v["b"].clone().requires_grad_(True)}
            for k, v in p.items()}
    y_ref = O.forward(leaf, x)
    loss_ref = ((y_ref - tgt) ** 2).mean()
    loss_ref.backward()
    # GPU kernels
    xg = O.from_nchw(x).cuda()
    tg = O.from_nchw(tgt).cuda()
    y = net.forward(xg, B)
    y_cpu = O.to_nchw(y.cpu(), B, H, W)
    rel = float((y_cpu - y_ref.detach()).norm() / y_ref.detach().norm())
    assert rel < 3e-2, rel
    dout = torch.empty_like(y)
    loss = torch.zeros(1, device="cuda")
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    _lib.call("amhd_nn_mse", y.data_ptr(), tg.data_ptr(), y.numel(), dout.data_ptr(), loss.data_ptr(), stream_ptr())
    assert abs(float(loss) - float(loss_ref.detach())) / float(loss_ref.detach()) < 3e-2
    net.backward(dout, B)
    worst = {}
    for s in net.specs:
        gw = net.p[s.name]["gw"].cpu().reshape(leaf[s.name]["w"].shape)
        gb = net.p[s.name]["gb"].cpu()
        rw = leaf[s.name]["w"].grad
        rb = leaf[s.name]["b"].grad
        worst[s.name] = (float((gw - rw).norm() / rw.norm().clamp_min(1e-30)),
                         float((gb - rb).norm() / rb.norm().clamp_min(1e-30)))
    bad = {k: v for k, v in worst.items() if max(v) > 6e-2}
    assert not bad, worst


def test_adam_matches_torch_adam():
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    g = torch.Generator().manual_seed(0)
    w0 = torch.randn(1000, generator=g)
    grads = [torch.randn(1000, generator=g) for _ in range(4)]
    wr = w0.clone().requires_grad_(True)
    opt = torch.optim.Adam([wr], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = w0.cuda(), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    for t, gr in enumerate(grads, 1):
        wr.grad = gr.clone()
        opt.step()
        gg = gr.cuda()
        _lib.call("amhd_nn_adam", w.data_ptr(), gg.data_ptr(), m.data_ptr(), v.data_ptr(), None, 1000, 1e-2, 0.9,
                  0.999, 1e-8, t, 0.0, stream_ptr())
    assert torch.allclose(w.cpu(), wr.detach(), atol=1e-6, rtol=1e-5)


def test_adam_multi_matches_torch_adam():
    """amhd_nn_adam_multi: three tensors of different sizes in one launch, the
    step scalars read from device memory, against torch.optim.Adam."""
    import ctypes
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    g = torch.Generator().manual_seed(1)
    sizes = (1000, 37, 70000)
    w0 = [torch.randn(n, generator=g) for n in sizes]
    refs = [w.clone().requires_grad_(True) for w in w0]
    opt = torch.optim.Adam(refs, lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    ws = [w.cuda() for w in w0]
    ms = [torch.zeros_like(w) for w in ws]
    vs = [torch.zeros_like(w) for w in ws]
    gs = [torch.zeros_like(w) for w in ws]
    table = (_lib.NNTensor * 3)()
    for r, w, gg, m, v in zip(table, ws, gs, ms, vs):
        r.w, r.g, r.m, r.v, r.w_bf16, r.n, r.weight_decay = w.data_ptr(), gg.data_ptr(), m.data_ptr(), v.data_ptr(), \
            None, w.numel(), 0.0
    tdev = torch.frombuffer(bytearray(bytes(table)), dtype=torch.uint8).cuda()
    hyper = torch.zeros(6, device="cuda")
    for t in range(1, 5):
        grads = [torch.randn(n, generator=g) for n in sizes]
        for r, gr in zip(refs, grads):
            r.grad = gr.clone()
        opt.step()
        for gg, gr in zip(gs, grads):
            gg.copy_(gr)
        hyper.copy_(torch.tensor([1e-2, 0.9, 0.999, 1e-8, 1 / (1 - 0.9 ** t), 1 / (1 - 0.999 ** t)]))
        _lib.call("amhd_nn_adam_multi", tdev.data_ptr(), 3, max(sizes), hyper.data_ptr(), stream_ptr())
    for w, r in zip(ws, refs):
        assert torch.allclose(w.cpu(), r.detach(), atol=1e-6, rtol=1e-5)


def test_graphed_training_step_matches_eager():
    """train_step_graphed (forward, loss, backward and Adam captured once as a
    CUDA graph, replayed with the batch copied in) follows train_step: the same
    kernels, so the losses agree to the rounding that split-K accumulation
    order leaves (1e-4 relative) over 12 steps on changing batches."""
    from aeromhd_cuda_b200.corrector import Corrector, architecture, init_params
    H, W, B = 32, 16, 4
    host = init_params(architecture(), seed=5)
    a, b = Corrector(H, W, params=host), Corrector(H, W, params=host)
    g = torch.Generator(device="cuda").manual_seed(9)
    la, lb = [], []
    for step in range(12):
        x = torch.randn((10, B * H * W), device="cuda", generator=g)
        tg = 0.1 * torch.tanh(x)
        la.append(float(a.train_step(x, tg, B, lr=1e-3).item()))
        lb.append(float(b.train_step_graphed(x, tg, B, lr=1e-3).item()))
    assert b.t == a.t == 12 and len(b._graphs) == 1
    for u, v in zip(la, lb):
        assert abs(u - v) <= 1e-4 * abs(u), (u, v)
    wa, wb = a.p["e1"]["w"], b.p["e1"]["w"]
    assert float((wa - wb).abs().max()) <= 1e-4 * float(wa.abs().max())


@pytest.mark.parametrize("C,B,H,W", [(3, 2, 5, 7), (10, 4, 32, 16), (16, 1, 8, 8), (8, 2, 16, 64), (5, 3, 6, 12)])
def test_im2col_col2im_bias_grad_against_torch(C, B, H, W):
    """The convolution helpers against torch: im2col3 (3x3, zero padding) as
    unfold, col2im3 as its adjoint (fold), bias_grad as a row sum (N both a
    multiple of 4 and not)."""
    import torch.nn.functional as Fn
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    g = torch.Generator(device="cuda").manual_seed(C * 100 + H)
    X = torch.randn((C, B, H, W), device="cuda", generator=g)
    N = B * H * W
    col = torch.empty((C * 9, N), dtype=torch.bfloat16, device="cuda")
    _lib.call("amhd_nn_im2col3", X.data_ptr(), C, B, H, W, col.data_ptr(), stream_ptr())
    ref = Fn.unfold(X.permute(1, 0, 2, 3), 3, padding=1)            # [B][C*9][H*W]
    ref = ref.permute(1, 0, 2).reshape(C * 9, N)
    assert torch.equal(col, ref.to(torch.bfloat16))
    dcol = torch.randn((C * 9, N), device="cuda", generator=g)
    dX = torch.empty((C, N), device="cuda")
    _lib.call("amhd_nn_col2im3", dcol.data_ptr(), C, B, H, W, dX.data_ptr(), stream_ptr())
    fold = Fn.fold(dcol.view(C * 9, B, H * W).permute(1, 0, 2), (H, W), 3, padding=1)   # [B][C][H][W]
    assert torch.allclose(dX.view(C, B, H, W), fold.permute(1, 0, 2, 3), atol=1e-5)
    for n in (N, N - 1):
        dY = torch.randn((C, n), device="cuda", generator=g)
        db = torch.empty(C, device="cuda")
        _lib.call("amhd_nn_bias_grad", dY.data_ptr(), C, n, db.data_ptr(), stream_ptr())
        assert torch.allclose(db, dY.double().sum(1).float(), atol=1e-3, rtol=1e-5)


def _shifted(t):
    """A copy of t that starts 4 bytes past a 16-byte boundary (the library's scalar kernels)."""
    buf = torch.empty(t.numel() + 4, dtype=t.dtype, device=t.device)
    v = buf[1:1 + t.numel()].view(t.shape)
    v.copy_(t)
    return v


@pytest.mark.parametrize("CB,H,W", [(6, 8, 16), (12, 32, 64), (3, 6, 10)])
def test_elementwise_helpers_vector_and_scalar_paths(CB, H, W):
    """Pooling, upsampling (and their gradients), bias + ReLU, the ReLU
    gradient, axpy and the bfloat16 cast: the several-values-per-thread
    kernels (16-byte aligned operands, rows a multiple of 4) give the same bits
    as the one-value-per-thread kernels (operands 4 bytes off), and both match
    torch."""
    import ctypes
    import torch.nn.functional as Fn
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import stream_ptr
    g = torch.Generator(device="cuda").manual_seed(CB * 7 + W)
    X = torch.randn((CB, H, W), device="cuda", generator=g)
    h, w = H // 2, W // 2

    def both(fn, out_shape, *ins):
        res = []
        for shift in (False, True):
            args = [_shifted(t) if shift else t.clone() for t in ins]
            out = torch.zeros(out_shape, device="cuda")
            out = _shifted(out) if shift else out
            fn(out, *args)
            res.append(out.clone())
        assert torch.equal(res[0], res[1])
        return res[0]

    pooled = both(lambda o, x: _lib.call("amhd_nn_pool2", x.data_ptr(), CB, H, W, o.data_ptr(), 0, stream_ptr()),
                  (CB, h, w), X)
    assert torch.allclose(pooled, Fn.avg_pool2d(X.unsqueeze(1), 2).squeeze(1), atol=1e-6)
    dP = torch.randn((CB, h, w), device="cuda", generator=g)
    dXp = both(lambda o, d: _lib.call("amhd_nn_pool2", d.data_ptr(), CB, H, W, o.data_ptr(), 1, stream_ptr()),
               (CB, H, W), dP)
    assert torch.equal(dXp, 0.25 * dP.repeat_interleave(2, 1).repeat_interleave(2, 2))
    Xs = torch.randn((CB, h, w), device="cuda", generator=g)
    up = both(lambda o, x: _lib.call("amhd_nn_up2", x.data_ptr(), CB, h, w, o.data_ptr(), 0, stream_ptr()),
              (CB, H, W), Xs)
    assert torch.equal(up, Xs.repeat_interleave(2, 1).repeat_interleave(2, 2))
    dU = torch.randn((CB, H, W), device="cuda", generator=g)
    dXs = both(lambda o, d: _lib.call("amhd_nn_up2", d.data_ptr(), CB, h, w, o.data_ptr(), 1, stream_ptr()),
               (CB, h, w), dU)
    assert torch.allclose(dXs, 4.0 * Fn.avg_pool2d(dU.unsqueeze(1), 2).squeeze(1), atol=1e-5)
    # bias + ReLU over [C][N], N = H * W per channel
    C, N = CB, H * W
    bias = torch.randn(C, device="cuda", generator=g)
    for relu in (0, 1):
        def ba(o, y):
            o.copy_(y)
            _lib.call("amhd_nn_bias_act", o.data_ptr(), bias.data_ptr(), C, N, relu, stream_ptr())
        Y = both(ba, (C, N), X.view(C, N))
        ref = X.view(C, N) + bias[:, None]
        assert torch.equal(Y, ref.clamp_min(0.0) if relu else ref)

    def rb(o, d, y):
        o.copy_(d)
        _lib.call("amhd_nn_relu_bwd", o.data_ptr(), y.data_ptr(), C * N, stream_ptr())
    Yr = torch.randn((C, N), device="cuda", generator=g)
    dY = torch.randn((C, N), device="cuda", generator=g)
    assert torch.equal(both(rb, (C, N), dY, Yr), torch.where(Yr > 0, dY, torch.zeros_like(dY)))

    def ax(o, y, x):
        o.copy_(y)
        _lib.call("amhd_nn_axpy", o.data_ptr(), x.data_ptr(), ctypes.c_float(0.37), C * N, stream_ptr())
    assert torch.allclose(both(ax, (C, N), dY, Yr), dY + 0.37 * Yr, atol=1e-6)
    for shift in (False, True):
        src = _shifted(X) if shift else X
        out = torch.empty(X.numel() + 8, dtype=torch.bfloat16, device="cuda")
        dst = out[4 if shift else 0:][:X.numel()]
        _lib.call("amhd_nn_cast_bf16", src.data_ptr(), dst.data_ptr(), X.numel(), stream_ptr())
        assert torch.equal(dst.view(X.shape), X.to(torch.bfloat16))


def test_restrict_pack_apply():
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import make_grid, padded_state, stream_ptr
    f = 4
    _, Uf = padded_state(64, 32, torch.float32)
    Uf.copy_(torch.randn(Uf.shape, device="cuda"))
    out = torch.empty((10, 16, 8), device="cuda")
    _lib.call("amhd_nn_restrict", make_grid(Uf, 1.4), Uf.data_ptr(), f, out.data_ptr(), 128, 0, 1, stream_ptr())
    ref = Uf[:, 2:-2, 2:-2].double().reshape(10, 16, 4, 8, 4).mean(dim=(2, 4))
    assert torch.allclose(out.double(), ref, atol=1e-6)
    _, Uc = padded_state(16, 8, torch.float64)
    Uc.copy_(torch.randn(Uc.shape, device="cuda", dtype=torch.float64))
    mean = torch.arange(10, device="cuda", dtype=torch.float32)
    istd = torch.full((10,), 0.5, device="cuda")
    x = torch.empty((10, 128), device="cuda")
    g = make_grid(Uc, 1.4)
    _lib.call("amhd_nn_pack", g, Uc.data_ptr(), mean.data_ptr(), istd.data_ptr(), x.data_ptr(), 128, 0, stream_ptr())
    assert torch.allclose(x.double(), ((Uc[:, 2:-2, 2:-2] - mean.double().view(10, 1, 1)) * 0.5).reshape(10, 128),
                          atol=1e-5)
    before = Uc.clone()
    y = torch.randn((10, 128), device="cuda")
    scale = torch.linspace(1, 2, 10, device="cuda")
    _lib.call("amhd_nn_apply", g, Uc.data_ptr(), scale.data_ptr(), y.data_ptr(), 128, 0, stream_ptr())
    exp = before[:, 2:-2, 2:-2] + (scale.view(10, 1) * y).double().reshape(10, 16, 8)
    assert torch.allclose(Uc[:, 2:-2, 2:-2], exp, atol=1e-5)
    assert torch.equal(Uc[:, :2], before[:, :2])   # ghosts untouched


def test_training_follows_the_cpu_oracle_trajectory():
    """40 Adam steps on a fixed batch: the loss curve of the GPU training step
    (BF16 GEMMs, FP32 masters) follows the one of the same network trained in
    float32 with PyTorch autograd + torch.optim.Adam on the CPU, from the same
    initial weights, within 10 % at every step, and both fall."""
    from aeromhd_cuda_b200.corrector import Corrector, architecture, init_params
    import nn_oracle as O
    torch.manual_seed(0)
    H, W, B, lr, steps = 32, 16, 4, 1e-3, 40
    x = torch.randn(B, 10, H, W)
    tgt = 0.3 * torch.tanh(x.roll(1, dims=2))       # a smooth learnable map
    host = init_params(architecture(), seed=2)
    net = Corrector(H, W, params=host, seed=2)
    xg, tg = O.from_nchw(x).cuda(), O.from_nchw(tgt).cuda()
    ours = [float(net.train_step(xg, tg, B, lr=lr).item()) for _ in range(steps)]
    ref_p = {k: {n: v.clone().requires_grad_(True) for n, v in d.items()} for k, d in host.items()}
    opt = torch.optim.Adam([t for d in ref_p.values() for t in d.values()], lr=lr, betas=(0.9, 0.999), eps=1e-8)
    ref = []
    for _ in range(steps):
        opt.zero_grad()
        loss = torch.mean((O.forward(ref_p, x) - tgt) ** 2)
        ref.append(float(loss.detach()))
        loss.backward()
        opt.step()
    print("loss GPU:", ours[::8], "CPU oracle:", ref[::8])
    assert ref[-1] < 0.8 * ref[0] and ours[-1] < 0.8 * ours[0]
    for a, r in zip(ours, ref):
        assert abs(a - r) <= 0.10 * r, (a, r)


def test_guarded_apply_keeps_cells_admissible():
    """amhd_nn_apply_guarded: equals amhd_nn_apply (alpha = 1) where every
    corrected cell stays admissible; a cell whose corrected density or pressure
    would drop below half keeps its state and is counted."""
    from aeromhd_cuda_b200 import _lib
    from aeromhd_cuda_b200._tensors import make_grid, stream_ptr
    torch.manual_seed(3)
    U = torch.zeros((10, 12, 20), dtype=torch.float64, device="cuda")
    U[0] = 1.0 + 0.1 * torch.rand(12, 20, device="cuda", dtype=torch.float64)
    U[1:4] = 0.1 * torch.randn(3, 12, 20, device="cuda", dtype=torch.float64)
    U[4:7] = 0.1 * torch.randn(3, 12, 20, device="cuda", dtype=torch.float64)
    U[7] = 2.0
    U[9] = U[0] * torch.rand(12, 20, device="cuda", dtype=torch.float64)
    g = make_grid(U, 1.4)
    y = 0.01 * torch.randn((10, 128), device="cuda")
    scale = torch.ones(10, device="cuda")
    a, b = U.clone(), U.clone()
    rej = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("amhd_nn_apply", g, a.data_ptr(), scale.data_ptr(), y.data_ptr(), 128, 0, stream_ptr())
    _lib.call("amhd_nn_apply_guarded", g, b.data_ptr(), scale.data_ptr(), y.data_ptr(), 128, 0, 1.0, 0.5,
              0, rej.data_ptr(), stream_ptr())
    assert int(rej.item()) == 0
    assert torch.allclose(a, b, rtol=0, atol=1e-6)       # float32 arithmetic of the correction in both
    # cell (3, 5) of the interior: density would fall to 30 %; cell (7, 1): pressure negative
    y2 = y.clone().view(10, 8, 16)
    y2[0, 3, 5] = -0.7 * float(U[0, 5, 7])
    y2[7, 7, 1] = -5.0
    c = U.clone()
    rej.zero_()
    _lib.call("amhd_nn_apply_guarded", g, c.data_ptr(), scale.data_ptr(), y2.data_ptr(), 128, 0, 1.0, 0.5,
              0, rej.data_ptr(), stream_ptr())
    assert int(rej.item()) == 2
    assert torch.equal(c[:, 5, 7], U[:, 5, 7]) and torch.equal(c[:, 9, 3], U[:, 9, 3])
    half = U.clone()
    _lib.call("amhd_nn_apply_guarded", g, half.data_ptr(), scale.data_ptr(), y.data_ptr(), 128, 0, 0.5, 0.5,
              0, None, stream_ptr())
    assert torch.allclose(half[:, 2:-2, 2:-2] - U[:, 2:-2, 2:-2], 0.5 * (a - U)[:, 2:-2, 2:-2], atol=1e-6)

    # scalar modes: 2 leaves rho C alone, 1 scales its correction by 4 C (1 - C)
    for mode in (1, 2):
        d = U.clone()
        _lib.call("amhd_nn_apply_guarded", g, d.data_ptr(), scale.data_ptr(), y.data_ptr(), 128, 0, 1.0, 0.5,
                  mode, None, stream_ptr())
        assert torch.allclose(d[:9], a[:9], rtol=0, atol=1e-6)
        if mode == 2:
            assert torch.equal(d[9], U[9])
        else:
            C = (U[9] / U[0]).clamp(0, 1)
            assert torch.allclose(d[9] - U[9], (a[9] - U[9]) * 4 * C * (1 - C), atol=1e-6)


def test_trained_corrector_gains_over_no_correction_on_held_out_seeds():
    """What the trained network gains over the method without it: coarse/fine
    pairs generated by the solver (coarse 64x16 vs fine 256x64 runs of the
    shocked-interface draws, one correction interval of 0.02 from the fine state
    restricted), trained on 8 seeds with the library's own kernels; on 4
    held-out seeds the corrected one-interval error is well below the error of
    applying no correction (the plain coarse step)."""
    from aeromhd_cuda_b200 import learned
    starts = tuple(round(0.1 * k, 10) for k in range(0, 8))
    X, Y, wall = learned.generate_pairs(range(12), t_starts=starts, nyc=16, log=None)
    assert torch.isfinite(X).all() and torch.isfinite(Y).all()
    net, norm, hist = learned.train(X, Y, range(8), range(8, 12), epochs=40, batch=8, lr=1e-3, log=None)
    base = hist["val_loss_zero_correction"]
    print("held-out loss per epoch (every 8th):", [round(v, 4) for v in hist["val_loss"][::8]], "no correction:", base)
    assert hist["val_loss"][-1] < 0.5 * base
