"""CPU restatement of the neural path-guiding model -- TEST INFRASTRUCTURE ONLY.

The reference renderer has no path guiding; this file states the model the CUDA kernels
(swpathtracer_b200/csrc/guiding.cu) implement, in numpy, so their forward pass, gradients and
optimiser step can be checked (forward against this file, gradients also against finite
differences of this file).

Model (all constants mirror csrc/guiding.cuh):
  * position -> multiresolution hash grid: L = 16 levels, F = 2 features per level, T = 2^19 entries
    per level, level resolution floor(16 * b^l + 1e-6) with b = exp(ln(1024/16) / (L-1)); a level with
    (N+1)^3 <= T is indexed densely, otherwise by the spatial hash
    (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T; trilinear weights of the 8 corners.
  * input u (48) = 32 grid features, normal (3), outgoing direction (3), 10 zeros.
  * MLP without biases: 48 -> 64 -> 64 -> 64 -> 64 (ReLU after each) -> 48 outputs (40 used).
  * output lobe k of 8: mu = normalize(y[5k:5k+3]), kappa = exp(clamp(y[5k+3], -2.3, 7)),
    weights = softmax(y[5k+4]); vMF pdf kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (mu.w - 1)}.
  * loss per record: -c * log q(w), c = the record's normalised weight; batch loss = mean.
  * Adam (beta1 0.9, beta2 0.99, eps 1e-15, bias-corrected); for the hash grid the lazy form:
    entries with a zero gradient keep their parameter and moments (adam_lazy).
BF16: the kernels round the MLP inputs of every layer and the weights to bf16 and accumulate in
fp32; bf16() below reproduces the rounding so the forward can be compared tightly.
"""
import numpy as np

L, F, T = 16, 2, 1 << 19
N_MIN, N_MAX = 16, 1024
IN, HID, OUT, LOBES = 48, 64, 48, 8
PRIMES = (1, 2654435761, 805459861)
KAPPA_LO, KAPPA_HI = -2.3, 7.0


def level_res(l):
    b = np.exp(np.log(N_MAX / N_MIN) / (L - 1))
    return int(np.floor(N_MIN * b ** l + 1e-6))


def bf16(x):
    """Round float32 to bfloat16 (nearest even) and back to float32."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def grid_index(l, ix, iy, iz):
    n = level_res(l) + 1
    if n ** 3 <= T:
        return (ix + iy * n + iz * n * n).astype(np.int64)
    h = (ix.astype(np.uint64) * np.uint64(PRIMES[0])) ^ (iy.astype(np.uint64) * np.uint64(PRIMES[1])) ^ \
        (iz.astype(np.uint64) * np.uint64(PRIMES[2]))
    return ((h & np.uint64(0xFFFFFFFF)) % np.uint64(T)).astype(np.int64)


def encode(table, xn):
    """table float32 [L, T, F] (bf16 values), xn [n, 3] in [0, 1] -> features [n, 32] and the
    (index, weight) of every corner for the backward pass."""
    xn = np.clip(xn, 0.0, 0.99999994)
    n = xn.shape[0]
    feats = np.zeros((n, L * F), np.float64)
    corners = []
    for l in range(L):
        res = level_res(l)
        p = xn * res
        p0 = np.floor(p)
        fr = p - p0
        p0 = p0.astype(np.int64)
        cl = []
        for c in range(8):
            dx, dy, dz = c & 1, (c >> 1) & 1, (c >> 2) & 1
            w = (fr[:, 0] if dx else 1 - fr[:, 0]) * (fr[:, 1] if dy else 1 - fr[:, 1]) * \
                (fr[:, 2] if dz else 1 - fr[:, 2])
            idx = grid_index(l, p0[:, 0] + dx, p0[:, 1] + dy, p0[:, 2] + dz)
            feats[:, l * F:(l + 1) * F] += w[:, None] * table[l, idx].astype(np.float64)
            cl.append((idx, w))
        corners.append(cl)
    return feats, corners


def inputs(feats, normal, wo):
    u = np.zeros((feats.shape[0], IN))
    u[:, :32] = feats
    u[:, 32:35] = normal
    u[:, 35:38] = wo
    return u


def forward(weights, u, emulate_bf16=True):
    """weights: [W0 (64x48), W1, W2, W3 (64x64), W4 (48x64)]; returns outputs and the per-layer inputs."""
    xs = []
    x = u
    for i, W in enumerate(weights):
        xin = bf16(x) if emulate_bf16 else x
        xs.append(xin.astype(np.float64))
        Wq = bf16(W) if emulate_bf16 else W
        z = xin.astype(np.float64) @ Wq.astype(np.float64).T
        x = np.maximum(z, 0.0) if i < len(weights) - 1 else z
    return x, xs


def decode(y):
    raw = y[:, :5 * LOBES].reshape(-1, LOBES, 5)
    m = raw[:, :, 0:3]
    mn = np.linalg.norm(m, axis=2, keepdims=True)
    mu = m / np.maximum(mn, 1e-12)
    r3 = np.clip(raw[:, :, 3], KAPPA_LO, KAPPA_HI)
    kappa = np.exp(r3)
    logits = raw[:, :, 4]
    e = np.exp(logits - logits.max(1, keepdims=True))
    w = e / e.sum(1, keepdims=True)
    return mu, kappa, w, mn, raw


def vmf_pdf(mu, kappa, wdir):
    c = (mu * wdir[:, None, :]).sum(2)
    norm = kappa / (2 * np.pi * (1 - np.exp(-2 * kappa)))
    return norm * np.exp(kappa * (c - 1))


def mixture_pdf(y, wdir):
    mu, kappa, w, _, _ = decode(y)
    return (w * vmf_pdf(mu, kappa, wdir)).sum(1)


def loss_and_grad_y(y, wdir, cw):
    """mean(-cw * log q); gradient wrt y (same shape as y)."""
    n = y.shape[0]
    mu, kappa, w, mn, raw = decode(y)
    f = vmf_pdf(mu, kappa, wdir)
    q = (w * f).sum(1)
    loss = np.mean(-cw * np.log(q))
    g = np.zeros_like(y)
    coef = (-cw / n)[:, None]                     # d loss / d log q
    r = w * f / q[:, None]                        # responsibility of each lobe
    gl = coef * (r - w)                           # logits
    c = (mu * wdir[:, None, :]).sum(2)
    e2 = np.exp(-2 * kappa)
    dlnC = 1.0 / kappa - 2 * e2 / (1 - e2)
    dk = coef * r * (dlnC + (c - 1))              # d/d kappa
    r3 = raw[:, :, 3]
    inside = (r3 > KAPPA_LO) & (r3 < KAPPA_HI)
    g3 = dk * kappa * inside
    gmu = (coef * r * kappa)[:, :, None] * wdir[:, None, :]
    gm = (gmu - (gmu * mu).sum(2, keepdims=True) * mu) / np.maximum(mn, 1e-12)
    gg = np.concatenate([gm, g3[:, :, None], gl[:, :, None]], 2).reshape(n, 5 * LOBES)
    g[:, :5 * LOBES] = gg
    return loss, g


def backward(weights, xs, gy, emulate_bf16=True):
    """Gradients of the weights and of the network input, given d loss / d y."""
    gws = [None] * len(weights)
    g = gy
    for i in reversed(range(len(weights))):
        W = bf16(weights[i]) if emulate_bf16 else weights[i]
        gws[i] = g.T @ xs[i]
        gx = g @ W.astype(np.float64)
        if i > 0:
            gx = gx * (xs[i] > 0)
        g = gx
    return gws, g


def grid_grad(corners, gfeat, shape):
    gt = np.zeros(shape, np.float64)
    for l in range(L):
        for idx, w in corners[l]:
            np.add.at(gt[l], idx, w[:, None] * gfeat[:, l * F:(l + 1) * F])
    return gt


def adam_lazy(p, g, m, v, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-15):
    """Adam where only entries with a nonzero gradient move (the hash grid's update)."""
    p2, m2, v2 = adam(p, g, m, v, step, lr, b1, b2, eps)
    touched = g != 0
    return np.where(touched, p2, p), np.where(touched, m2, m), np.where(touched, v2, v)


def adam(p, g, m, v, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-15):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
