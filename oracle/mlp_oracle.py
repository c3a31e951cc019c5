"""CPU oracle of the learned-truncation network (test infrastructure only).

The network maps the 16 term features to a predicted log10 |contribution|:
    Z1 = bf16(X) @ bf16(W1)^T + b1,  H1 = GELU(Z1)
    Z2 = bf16(H1) @ bf16(W2)^T + b2, H2 = GELU(Z2)
    y  = H2 . bf16(w3) + b3
with GELU(x) = x * Phi(x) (exact, erf form) and loss = mean((y - t)^2).
The GPU kernels multiply bf16 operands on the tensor cores with FP32
accumulation; this restatement rounds the same operands to bf16 (round to
nearest even) and accumulates in float64, so the two agree to FP32 rounding of
the sums (plus the rare bf16 rounding flip such a difference causes).

The reference (PauliOperators.jl) has no learned truncation; this oracle checks
the kernels against the mathematics of the network and its gradients, and
`fd_check` checks the analytic backward pass here against central differences.

Parameter vector layout (5,313 FP32 values), shared with the device:
    W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3[1]
"""
import math

import numpy as np

F_IN, H = 16, 64
SIZES = [("W1", (H, F_IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,)), ("b3", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)   # 5313


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), via the float32 value."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(f)
    r = r.astype(np.uint32).view(np.float32).astype(np.float64)
    if np.any(nan):
        r[nan] = np.nan
    return r


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def init_params(seed):
    """He-style initialisation from a seeded generator."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0.0, math.sqrt(2.0 / F_IN), (H, F_IN)), "b1": np.zeros(H),
         "W2": rng.normal(0.0, math.sqrt(2.0 / H), (H, H)), "b2": np.zeros(H),
         "w3": rng.normal(0.0, math.sqrt(1.0 / H), H), "b3": np.zeros(1)}
    return pack(d).astype(np.float32).astype(np.float64)


def forward(p, X, rounding=True):
    """Returns y and the intermediates (Z1, H1, Z2, H2, operands)."""
    d = unpack(p)
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    Xb = r(X)
    W1, W2, w3 = r(d["W1"]), r(d["W2"]), r(d["w3"])
    Z1 = Xb @ W1.T + d["b1"]
    H1 = gelu(Z1)
    H1b = r(H1)
    Z2 = H1b @ W2.T + d["b2"]
    H2 = gelu(Z2)
    y = H2 @ w3 + d["b3"][0]
    return y, dict(Xb=Xb, W1=W1, W2=W2, w3=w3, Z1=Z1, H1b=H1b, Z2=Z2, H2=H2)


def loss_grad(p, X, t, rounding=True):
    """mean((y - t)^2) and its gradient with respect to the FP32 master parameters
    (straight-through the bf16 rounding of the weights)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    y, c = forward(p, X, rounding)
    B = len(y)
    dy = 2.0 * (y - t) / B
    dw3 = c["H2"].T @ dy
    db3 = np.array([dy.sum()])
    dZ2 = np.outer(dy, c["w3"]) * gelu_grad(c["Z2"])
    dZ2b = r(dZ2)
    dW2 = dZ2b.T @ c["H1b"]
    db2 = dZ2.sum(axis=0)
    dH1 = dZ2b @ c["W2"]
    dZ1 = dH1 * gelu_grad(c["Z1"])
    dZ1b = r(dZ1)
    dW1 = dZ1b.T @ c["Xb"]
    db1 = dZ1.sum(axis=0)
    g = pack(dict(W1=dW1, b1=db1, W2=dW2, b2=db2, w3=dw3, b3=db3))
    return float(np.mean((y - t) ** 2)), g


def fd_check(seed=0, n=37, eps=1e-6):
    """Max relative difference between the analytic gradient (no rounding) and
    central differences of the loss, over all 5,313 parameters."""
    rng = np.random.default_rng(seed)
    p = init_params(seed)
    X = rng.normal(0.0, 1.0, (n, F_IN))
    t = rng.normal(0.0, 1.0, n)
    _, g = loss_grad(p, X, t, rounding=False)
    num = np.zeros_like(p)
    for i in range(len(p)):
        q = p.copy(); q[i] += eps
        lp, _ = loss_grad(q, X, t, rounding=False)
        q[i] -= 2 * eps
        lm, _ = loss_grad(q, X, t, rounding=False)
        num[i] = (lp - lm) / (2 * eps)
    return float(np.abs(num - g).max() / max(1e-12, np.abs(g).max()))


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015) in float64."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def term_features(ctx, z, x, c):
    """The 16 term features (float32), restated from their definition: ctx is a
    pp_feature_ctx (nbr, light_cone, boundary, row, col, layer_frac,
    remaining_frac, theta_j, theta_h); z, x are the term's 64-bit words."""
    z, x = int(z), int(x)
    s = z | x
    pc = lambda v: bin(v).count("1")
    ac = abs(float(c))
    lg = math.log10(ac) if ac > 0.0 else -300.0
    f = np.zeros(16, dtype=np.float32)
    f[0] = np.float32(max((lg + 3.0) / 3.0, -4.0))
    w12 = np.float32(1.0) / np.float32(12.0)
    f[1] = np.float32(pc(x & ~z)) * w12
    f[2] = np.float32(pc(x & z)) * w12
    f[3] = np.float32(pc(z & ~x)) * w12
    f[4] = np.float32(pc(s)) * w12
    f[5] = np.float32(pc(s & int(ctx.light_cone))) * w12
    f[6] = np.float32(ctx.layer_frac)
    f[7] = np.float32(ctx.remaining_frac)
    qs = [q for q in range(64) if (s >> q) & 1]
    pairs = sum(pc(int(ctx.nbr[q]) & s) for q in qs) // 2
    xpairs = sum(pc(int(ctx.nbr[q]) & x) for q in qs if (x >> q) & 1) // 2
    comps, rem = 0, s
    while rem:
        comp = rem & -rem
        prev = 0
        while comp != prev:
            prev = comp
            for q in range(64):
                if (comp >> q) & 1:
                    comp |= int(ctx.nbr[q]) & s
        rem &= ~comp
        comps += 1
    f[8] = np.float32(pairs) * w12
    f[9] = np.float32(comps) * w12
    if qs:
        rows = [ctx.row[q] for q in qs]
        cols = [ctx.col[q] for q in qs]
        f[10] = np.float32(max(rows) - min(rows) + 1) * np.float32(0.125)
        f[11] = np.float32(max(cols) - min(cols) + 1) * np.float32(0.125)
    f[12] = np.float32(pc(s & int(ctx.boundary))) * w12
    f[13] = np.float32(xpairs) * w12
    f[14] = np.float32(ctx.theta_j) * np.float32(2.0)
    f[15] = np.float32(ctx.theta_h) * np.float32(2.0)
    return f


def fkey(score):
    """Ordered 32-bit key of float32 scores (larger score, larger key)."""
    u = np.asarray(score, dtype=np.float32).view(np.uint32).astype(np.uint64)
    neg = (u >> 31) == 1
    return np.where(neg, (~u) & 0xFFFFFFFF, u | 0x80000000)


def budget_select(scores, budget):
    """Indices (in order) of the `budget` largest scores; ties at the cut keep the
    smaller index (the smaller key of a sorted vector)."""
    k = fkey(scores)
    n = len(k)
    if n <= budget:
        return np.arange(n)
    order = np.lexsort((np.arange(n), -k.astype(np.int64)))
    return np.sort(order[:budget])
