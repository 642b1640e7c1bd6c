"""CPU float32 oracle of the corrector network (PyTorch autograd on the CPU).

TEST INFRASTRUCTURE ONLY: the GPU kernels' forward pass and gradients are
checked against this.  Same architecture as aeromhd_cuda_b200.corrector:
3x3 zero-padded convolutions, 2x2 average pooling, nearest 2x upsampling,
1x1 convolutions with additive skips, ReLU after every 3x3 except the last.
"""
import torch
import torch.nn.functional as F


def forward(params, x):
    """params: {name: {"w": [Cout,Cin,k,k], "b": [Cout]}} (requires_grad as wanted); x: [B,10,H,W]."""
    def conv(name, t, relu):
        w, b = params[name]["w"], params[name]["b"]
        y = F.conv2d(t, w, b, padding=w.shape[-1] // 2)
        return F.relu(y) if relu else y

    e1 = conv("e1", x, True)
    e2 = conv("e2", F.avg_pool2d(e1, 2), True)
    e3 = conv("e3", F.avg_pool2d(e2, 2), True)
    e4 = conv("e4", F.avg_pool2d(e3, 2), True)
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")
    d3 = conv("d3", conv("d3a", up(e4), False) + e3, True)
    d2 = conv("d2", conv("d2a", up(d3), False) + e2, True)
    d1 = conv("d1", conv("d1a", up(d2), False) + e1, True)
    return conv("out", d1, False)


def to_nchw(a, B, H, W):
    """[C][B*H*W] -> [B][C][H][W]"""
    C = a.shape[0]
    return a.reshape(C, B, H, W).permute(1, 0, 2, 3).contiguous()


def from_nchw(t):
    B, C, H, W = t.shape
    return t.permute(1, 0, 2, 3).reshape(C, B * H * W).contiguous()
