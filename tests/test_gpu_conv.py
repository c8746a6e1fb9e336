"""The tensor-core 3x3x3 convolution (smoke_b200_conv3d_cuda) against a float64 convolution of the same BF16
inputs and weights. Channel 0 is also written in FP32, which isolates the accumulation (FP32 sums of exact BF16
products: normwise error ~1e-6); the BF16 output adds one rounding per value (2^-9 relative)."""
import ctypes as C

import numpy as np
import pytest
import torch

import smoke_abi as abi

pytestmark = pytest.mark.gpu

# the network's forward layers (2->16 ... 16->1) and a few other shapes (output channels that need several
# chunks of 16 or 32, odd channel counts); the backward-data convolutions are covered by the gradient tests
LAYERS = [(2, 16), (16, 32), (32, 64), (64, 128), (128, 64), (64, 32), (32, 16), (16, 1), (8, 1), (5, 3), (20, 40), (64, 16)]


def store(c):
    return 8 if c <= 8 else ((c + 15) // 16) * 16


def reference(x, w, b, relu):
    """x: [nz, ny, nx, cin] float64, w: [27, cin, cout] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)), b: [cout]."""
    nz, ny, nx, cin = x.shape
    cout = w.shape[2]
    xp = np.zeros((nz + 2, ny + 2, nx + 2, cin))
    xp[1:-1, 1:-1, 1:-1] = x
    out = np.zeros((nz, ny, nx, cout))
    for tap in range(27):
        dx, dy, dz = tap % 3 - 1, (tap // 3) % 3 - 1, tap // 9 - 1
        out += xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx] @ w[tap]
    out += b
    return np.maximum(out, 0.0) if relu else out


def bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)


def run(lib, shape, cin, cout, relu, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = np.zeros((nz, ny, nx, store(cin)), np.float32)
    x[..., :cin] = rng.standard_normal((nz, ny, nx, cin))
    w = (rng.standard_normal((27, cin, cout)) / np.sqrt(27 * cin)).astype(np.float32)
    b = (rng.standard_normal(cout) * 0.1).astype(np.float32)
    xb, wb = bf16(x), bf16(w)
    x_dev = xb.cuda().contiguous()
    w_dev = torch.from_numpy(w).cuda()  # FP32 [27][cin][cout]
    b_dev = torch.from_numpy(b).cuda()
    assert w_dev.dtype == torch.float32 and b_dev.dtype == torch.float32
    out = torch.zeros((nz, ny, nx, store(cout)), dtype=torch.bfloat16, device="cuda")
    out0 = torch.zeros((nz, ny, nx), dtype=torch.float32, device="cuda")
    fn = lib.smoke_b200_conv3d_cuda
    fn.argtypes = [C.c_int] * 5 + [C.c_void_p] * 3 + [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    s = torch.cuda.current_stream()
    code = fn(nx, ny, nz, cin, cout, x_dev.data_ptr(), w_dev.data_ptr(), b_dev.data_ptr(), int(relu), out.data_ptr(), out0.data_ptr(), C.c_void_p(s.cuda_stream))
    assert code == abi.RESULT_OK
    torch.cuda.synchronize()
    ref = reference(xb.float().numpy()[..., :cin].astype(np.float64), wb.float().numpy().astype(np.float64), b.astype(np.float64), relu)
    return out.float().cpu().numpy(), out0.cpu().numpy(), ref


@pytest.mark.parametrize("cin,cout", LAYERS, ids=[f"{a}to{b}" for a, b in LAYERS])
@pytest.mark.parametrize("relu", [False, True], ids=["linear", "relu"])
def test_conv3d_matches_float64(smoke_lib, cin, cout, relu):
    got, got0, ref = run(smoke_lib.lib, (21, 13, 11), cin, cout, relu, seed=cin * 100 + cout)
    scale = np.abs(ref).max()
    # FP32 accumulation of K = 27 x cin products: the rounding grows like sqrt(K) (2e-6 at K <= 216)
    k = 27 * store(cin)
    assert np.abs(got0 - ref[..., 0]).max() <= 2e-6 * max(1.0, np.sqrt(k / 216.0)) * scale
    assert np.abs(got[..., :cout] - ref).max() <= 8e-3 * scale
    assert not got[..., cout:].any()  # stored channels past cout are 0


@pytest.mark.parametrize("shape", [(1, 1, 1), (128, 1, 1), (129, 3, 2), (5, 7, 130), (64, 64, 33)])
def test_conv3d_shapes(smoke_lib, shape):
    got, got0, ref = run(smoke_lib.lib, shape, 8, 16, False, seed=7)
    scale = np.abs(ref).max()
    assert np.abs(got0 - ref[..., 0]).max() <= 2e-6 * scale
    assert np.abs(got - ref).max() <= 8e-3 * scale
