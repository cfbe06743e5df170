"""Oracle (test infrastructure only): numpy forward and backward of the
scatter-surrogate U-Net of ggems_b200/csrc/gg_unet.cu, same architecture and
flat parameter layout, in float64.  Used by the tests to check the GPU
kernels' outputs and gradients (which run in BF16 with FP32 accumulation),
and itself checked against finite differences.  There is no reference
counterpart: GGEMS has no learned component, so this is the only checker.

Parameter layout: for each of the 14 3x3 layers, W[tap][cout][cin] then
b[cout]; then the 1x1 output layer w[32], b[1].

Input stage: the 2 input maps (a, b) become 10 of the first layer's 16
channels -- a, b, box means of a and of b over (2r+1)^2 windows (r = 4, 16,
64; zero outside the image, divided by the full window area) and the means of
a and b over the whole image.
"""

import numpy as np

SPEC = [(16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 128, 4), (128, 128, 4), (128, 256, 8),
        (256, 256, 8), (384, 128, 4), (128, 128, 4), (192, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1)]


def unpack(params):
    layers, off = [], 0
    for cin, cout, _ in SPEC:
        w = params[off:off + 9 * cin * cout].reshape(9, cout, cin)
        off += 9 * cin * cout
        b = params[off:off + cout]
        off += cout
        layers.append((w, b))
    wo = params[off:off + 32]
    bo = params[off + 32:off + 33]
    return layers, wo, bo, off + 33


def parameter_count():
    return unpack(np.zeros(10 ** 7))[3]


def _shift(x, dy, dx):
    """x [B,H,W,C] shifted so that out[y,x] = x[y+dy, x+dx] (zero outside)."""
    B, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    out[:, ys:ye, xs:xe] = x[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def conv3x3(x, w):
    """y[p][co] = sum_tap sum_ci x[p + off(tap)][ci] w[tap][co][ci]."""
    y = 0.0
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        y = y + np.einsum("bhwc,oc->bhwo", _shift(x, ky - 1, kx - 1), w[tap])
    return y


def conv3x3_backward(x, w, dy):
    dw = np.zeros_like(w)
    dx = np.zeros_like(x)
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        xs = _shift(x, ky - 1, kx - 1)
        dw[tap] = np.einsum("bhwo,bhwc->oc", dy, xs)
        dx += _shift(np.einsum("bhwo,oc->bhwc", dy, w[tap]), 1 - ky, 1 - kx)
    return dx, dw


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def pool_backward(dy):
    return np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_backward(dy):
    B, H, W, C = dy.shape
    return dy.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


CONTEXT_RADII = (4, 16, 64)
INPUT_CHANNELS = 2 + 2 * len(CONTEXT_RADII) + 2


def box_mean(img, r):
    """[B,S,S] -> window sums over (2r+1)^2 (zero padded) / (2r+1)^2."""
    B, S, _ = img.shape
    I = np.zeros((B, S + 1, S + 1))
    I[:, 1:, 1:] = img.cumsum(1).cumsum(2)
    lo = np.clip(np.arange(S) - r, 0, S)
    hi = np.clip(np.arange(S) + r + 1, 0, S)
    s = I[:, hi][:, :, hi] - I[:, lo][:, :, hi] - I[:, hi][:, :, lo] + I[:, lo][:, :, lo]
    return s / float((2 * r + 1) ** 2)


def input_stage(inp):
    """[B,S,S,2] -> [B,S,S,16] first-layer input."""
    B, S, _, _ = inp.shape
    x0 = np.zeros((B, S, S, 16))
    x0[..., :2] = inp
    for m in range(2):
        for k, r in enumerate(CONTEXT_RADII):
            x0[..., 2 + 3 * m + k] = box_mean(inp[..., m], r)
        x0[..., 8 + m] = inp[..., m].mean(axis=(1, 2))[:, None, None]
    return x0


def forward(params, inp):
    """inp [B,S,S,2] -> (output [B,S,S], cache)."""
    layers, wo, bo, _ = unpack(params)
    x0 = input_stage(np.asarray(inp, np.float64))
    acts, ins = [], []

    def conv(i, x):
        w, b = layers[i]
        a = np.maximum(conv3x3(x, w) + b, 0.0)
        ins.append(x)
        acts.append(a)
        return a

    a1 = conv(1, conv(0, x0))
    a3 = conv(3, conv(2, pool(a1)))
    a5 = conv(5, conv(4, pool(a3)))
    a7 = conv(7, conv(6, pool(a5)))
    a9 = conv(9, conv(8, np.concatenate([up(a7), a5], axis=-1)))
    a11 = conv(11, conv(10, np.concatenate([up(a9), a3], axis=-1)))
    a13 = conv(13, conv(12, np.concatenate([up(a11), a1], axis=-1)))
    y = a13 @ wo + bo[0]
    return y, (ins, acts)


def loss_and_gradients(params, inp, target):
    layers, wo, bo, n = unpack(params)
    y, (ins, acts) = forward(params, inp)
    N = y.size
    diff = y - target
    loss = float((diff ** 2).sum() / N)
    grads = np.zeros(n)
    g_layers, gwo, gbo, _ = unpack(grads)
    dy = 2.0 * diff / N
    gwo[:] = np.einsum("bhw,bhwc->c", dy, acts[13])
    gbo[0] = dy.sum()
    dact = {13: dy[..., None] * wo}
    skip = {}

    def conv_back(i):
        w, _ = layers[i]
        dpre = dact[i] * (acts[i] > 0)
        dx, dw = conv3x3_backward(ins[i], w, dpre)
        g_layers[i][0][:] = dw
        g_layers[i][1][:] = dpre.sum(axis=(0, 1, 2))
        return dx

    for i in (13,):
        dact[12] = conv_back(13)
    dc = conv_back(12)
    dact[11], skip[1] = up_backward(dc[..., :64]), dc[..., 64:]
    dact[10] = conv_back(11)
    dc = conv_back(10)
    dact[9], skip[3] = up_backward(dc[..., :128]), dc[..., 128:]
    dact[8] = conv_back(9)
    dc = conv_back(8)
    dact[7], skip[5] = up_backward(dc[..., :256]), dc[..., 256:]
    dact[6] = conv_back(7)
    dact[5] = skip[5] + pool_backward(conv_back(6))
    dact[4] = conv_back(5)
    dact[3] = skip[3] + pool_backward(conv_back(4))
    dact[2] = conv_back(3)
    dact[1] = skip[1] + pool_backward(conv_back(2))
    dact[0] = conv_back(1)
    conv_back(0)
    return loss, grads
