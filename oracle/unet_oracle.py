"""FP64 oracle of the learned preconditioner's network. Test infrastructure: only tests/ import it; the library never
runs it.

The reference has no learned preconditioner, so there is no reference file to follow: this restates the library's own
network (unet.h, unet.cu) in numpy float64, forward and backward (hand-written, no autograd), for the gradient check
of the tensor-core kernels. With `emulate=True` the values the GPU stores in BF16 (weights, activations, activation
gradients) are rounded to BF16 at the same points, which leaves only FP32-versus-FP64 summation differences.

Network: level 0 is the volume, level l + 1 halves each extent of level l (rounding up); channels 16, 32, 64, 128.
    e0 = relu(conv_a([r s, fluid]))      p1 = pool(e0)      e1 = relu(conv_b(p1))      p2 = pool(e1)
    e2 = relu(conv_c(p2))                p3 = pool(e2)      e3 = relu(conv_d(p3))      m3 = relu(conv_m(e3))
    s2 = up(m3) + e2                     u2 = relu(conv_e(s2))                         s1 = up(u2) + e1
    u1 = relu(conv_f(s1))                s0 = up(u1) + e0   y = conv_g(s0)             N(r) = fluid * y / s,
with s = sqrt(n) / ||r||. Loss of one sample: L = sum_fluid (y - s t)^2 / (s^2 sum_fluid t^2).
"""
import numpy as np

# (cin, cout, level) per layer, in execution order: a, b, c, d, m, e, f, g
LAYERS = [(2, 16, 0), (16, 32, 1), (32, 64, 2), (64, 128, 3), (128, 64, 3), (64, 32, 2), (32, 16, 1), (16, 1, 0)]


def param_count():
    return sum(27 * ci * co + co for ci, co, _ in LAYERS)


def unpack(params):
    """[(W [27, cin, cout], b [cout])] per layer from the flat parameter vector (weights then biases per layer)."""
    out, o = [], 0
    p = np.asarray(params, np.float64)
    for ci, co, _ in LAYERS:
        w = p[o:o + 27 * ci * co].reshape(27, ci, co)
        o += 27 * ci * co
        b = p[o:o + co]
        o += co
        out.append((w, b))
    return out


def pack(grads):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in grads])


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a32 = np.ascontiguousarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _offsets():
    for tap in range(27):
        yield tap, tap % 3 - 1, (tap // 3) % 3 - 1, tap // 9 - 1


def conv(x, w, b=None):
    """out[q] = sum_tap x[q + offset(tap)] @ w[tap] (+ b), zero padding; x [nz, ny, nx, cin]."""
    nz, ny, nx, _ = x.shape
    xp = np.zeros((nz + 2, ny + 2, nx + 2, x.shape[3]))
    xp[1:-1, 1:-1, 1:-1] = x
    out = np.zeros((nz, ny, nx, w.shape[2]))
    for tap, dx, dy, dz in _offsets():
        out += xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx] @ w[tap]
    return out if b is None else out + b


def conv_data(g, w):
    """Gradient of conv with respect to its input: dx[q] = sum_tap g[q - offset(tap)] @ w[tap]^T."""
    nz, ny, nx, _ = g.shape
    gp = np.zeros((nz + 2, ny + 2, nx + 2, g.shape[3]))
    gp[1:-1, 1:-1, 1:-1] = g
    out = np.zeros((nz, ny, nx, w.shape[1]))
    for tap, dx, dy, dz in _offsets():
        out += gp[1 - dz:1 - dz + nz, 1 - dy:1 - dy + ny, 1 - dx:1 - dx + nx] @ w[tap].T
    return out


def conv_weight(x, g):
    """Gradient of conv with respect to (w, b): dw[tap] = sum_q x[q + offset(tap)]^T g[q], db = sum_q g[q]."""
    nz, ny, nx, ci = x.shape
    xp = np.zeros((nz + 2, ny + 2, nx + 2, ci))
    xp[1:-1, 1:-1, 1:-1] = x
    gf = g.reshape(-1, g.shape[3])
    dw = np.zeros((27, ci, g.shape[3]))
    for tap, dx, dy, dz in _offsets():
        dw[tap] = xp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx].reshape(-1, ci).T @ gf
    return dw, gf.sum(0)


def coarse_shape(shape):
    return tuple((v + 1) // 2 for v in shape)


def _counts(fine):
    """Children of each coarse cell (1..8) along each axis and in total."""
    cz, cy, cx = coarse_shape(fine)
    nz, ny, nx = fine
    kz = np.minimum(2, nz - 2 * np.arange(cz))
    ky = np.minimum(2, ny - 2 * np.arange(cy))
    kx = np.minimum(2, nx - 2 * np.arange(cx))
    return (kz[:, None, None] * ky[None, :, None] * kx[None, None, :]).astype(np.float64)


def up(c, fine):
    nz, ny, nx = fine
    z, y, x = np.arange(nz) // 2, np.arange(ny) // 2, np.arange(nx) // 2
    return c[z][:, y][:, :, x]


def up_adjoint(g, coarse):
    """Sum of the children's values into each parent (the gradient of up)."""
    out = np.zeros(coarse + (g.shape[3],))
    nz, ny, nx = g.shape[:3]
    np.add.at(out, (np.arange(nz)[:, None, None] // 2, np.arange(ny)[None, :, None] // 2, np.arange(nx)[None, None, :] // 2), g)
    return out


def pool(f):
    fine = f.shape[:3]
    return up_adjoint(f, coarse_shape(fine)) / _counts(fine)[..., None]


def pool_adjoint(gc, fine):
    """Each child receives its parent's gradient divided by the parent's children count."""
    return up(gc / _counts(fine)[..., None], fine)


def forward(params, r, occ, emulate=False):
    """Activations of one evaluation; r float [nz, ny, nx], occ uint8 (nonzero = solid)."""
    rnd = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    f32 = (lambda a: np.asarray(a, np.float32).astype(np.float64)) if emulate else (lambda a: np.asarray(a, np.float64))
    layers = [(rnd(w), f32(b)) for w, b in unpack(params)]  # BF16 weights, FP32 biases on the GPU
    r = np.asarray(r, np.float64)
    fluid = (np.asarray(occ) == 0).astype(np.float64)
    n = r.size
    nn = float(np.sum(np.asarray(r, np.float32).astype(np.float64) ** 2))
    s = float(np.float32(np.sqrt(n / nn))) if nn > 0 else 0.0
    x0 = np.stack([rnd(np.float32(r) * np.float32(s)), fluid], axis=-1)
    relu = lambda a: np.maximum(a, 0.0)
    A = {"s": s, "fluid": fluid, "x0": x0, "layers": layers}
    A["e0"] = rnd(relu(conv(x0, *layers[0])))
    A["p1"] = rnd(pool(A["e0"]))
    A["e1"] = rnd(relu(conv(A["p1"], *layers[1])))
    A["p2"] = rnd(pool(A["e1"]))
    A["e2"] = rnd(relu(conv(A["p2"], *layers[2])))
    A["p3"] = rnd(pool(A["e2"]))
    A["e3"] = rnd(relu(conv(A["p3"], *layers[3])))
    A["m3"] = rnd(relu(conv(A["e3"], *layers[4])))
    A["s2"] = rnd(up(A["m3"], A["e2"].shape[:3]) + A["e2"])
    A["u2"] = rnd(relu(conv(A["s2"], *layers[5])))
    A["s1"] = rnd(up(A["u2"], A["e1"].shape[:3]) + A["e1"])
    A["u1"] = rnd(relu(conv(A["s1"], *layers[6])))
    A["s0"] = rnd(up(A["u1"], A["e0"].shape[:3]) + A["e0"])
    A["y"] = conv(A["s0"], *layers[7])[..., 0]
    return A


def apply(params, r, occ, emulate=False):
    A = forward(params, r, occ, emulate)
    return A["fluid"] * A["y"] / A["s"] if A["s"] > 0 else np.zeros_like(A["y"])


def loss_and_gradient(params, r, occ, target, emulate=False):
    """(L, dL/dparams) of one sample, the gradient in the flat parameter layout."""
    rnd = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    A = forward(params, r, occ, emulate)
    s, fluid, L = A["s"], A["fluid"], A["layers"]
    t = np.asarray(target, np.float64) * fluid
    denom = s * s * float(np.sum(t * t))
    e = fluid * (A["y"] - s * t)
    loss = float(np.sum(e * e) / denom)
    gy = rnd(2.0 * e / denom)[..., None]
    grads = [None] * len(LAYERS)
    # g: y = conv_g(s0), s0 = up(u1) + e0
    grads[7] = conv_weight(A["s0"], gy)
    gs0 = rnd(conv_data(gy, L[7][0]))
    # f: u1 = relu(conv_f(s1)), s1 = up(u2) + e1
    gu1 = rnd(up_adjoint(gs0, A["u1"].shape[:3]) * (A["u1"] > 0))
    grads[6] = conv_weight(A["s1"], gu1)
    gs1 = rnd(conv_data(gu1, L[6][0]))
    # e: u2 = relu(conv_e(s2)), s2 = up(m3) + e2
    gu2 = rnd(up_adjoint(gs1, A["u2"].shape[:3]) * (A["u2"] > 0))
    grads[5] = conv_weight(A["s2"], gu2)
    gs2 = rnd(conv_data(gu2, L[5][0]))
    # m: m3 = relu(conv_m(e3)); e3 feeds m only
    gm3 = rnd(up_adjoint(gs2, A["m3"].shape[:3]) * (A["m3"] > 0))
    grads[4] = conv_weight(A["e3"], gm3)
    ge3 = rnd(conv_data(gm3, L[4][0]) * (A["e3"] > 0))
    # d: e3 = relu(conv_d(p3)), p3 = pool(e2)
    grads[3] = conv_weight(A["p3"], ge3)
    gp3 = rnd(conv_data(ge3, L[3][0]))
    # c: e2 feeds p3 and s2
    ge2 = rnd((gs2 + pool_adjoint(gp3, A["e2"].shape[:3])) * (A["e2"] > 0))
    grads[2] = conv_weight(A["p2"], ge2)
    gp2 = rnd(conv_data(ge2, L[2][0]))
    # b: e1 feeds p2 and s1
    ge1 = rnd((gs1 + pool_adjoint(gp2, A["e1"].shape[:3])) * (A["e1"] > 0))
    grads[1] = conv_weight(A["p1"], ge1)
    gp1 = rnd(conv_data(ge1, L[1][0]))
    # a: e0 feeds p1 and s0
    ge0 = rnd((gs0 + pool_adjoint(gp1, A["e0"].shape[:3])) * (A["e0"] > 0))
    grads[0] = conv_weight(A["x0"], ge0)
    return loss, pack(grads)


def initial_like(seed, scale=1.0):
    """Random parameters for tests (He-normal weights, small random biases)."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co, _ in LAYERS:
        out.append(rng.standard_normal(27 * ci * co) * np.sqrt(2.0 / (27 * ci)) * scale)
        out.append(rng.standard_normal(co) * 0.05)
    return np.concatenate(out).astype(np.float32)
