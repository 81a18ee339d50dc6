"""CPU restatement of the learned guiding network (numpy, float64).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the tensor-core kernels in
lambent_b200/csrc/guide_net.cu; the product never imports it.

The network has no counterpart in the reference (its guiding is the Markov-chain cache of
src/path_tracing/general.wesl:764-866), so this module restates the specification the CUDA code
implements, independently of it:

* 64 input features per query: the position normalised to the scene box, encoded as sin/cos of
  2^k pi u for k = 0..4 (30), the normal and outgoing direction (6), their sin/cos of 2^k pi v for
  k = 0..1 (24), three zeros and the constant 1.
* Four 64 x 64 layers Z = X W^T.  Column 63 of every layer input is 1 (so W[l][:, 63] is the bias);
  hidden outputs are ReLU'd and unit 63 is replaced by the constant 1.
* Head (40 outputs): logits 0-7 (softmax mixture weights), log-concentrations 8-15 (clamped to
  [-3, 6], exponentiated), lobe means 16-23 / 24-31 / 32-39 (x / y / z, normalised).
* vMF density kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu . w - 1)); loss -weight log q(w).

`bf16=True` rounds the features, weights, activations and head gradients to bfloat16 (round to
nearest even) where the kernels keep them in bfloat16; products accumulate in float64 here and in
float32 on the tensor cores.
"""
import numpy as np

WIDTH = 64
LAYERS = 4
OUT = 40
LOBES = 8
PARAMS = LAYERS * WIDTH * WIDTH
KAPPA_LOG_MIN, KAPPA_LOG_MAX = -3.0, 6.0


def bf16(x):
    """Round float values to bfloat16 (round to nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    nan = np.isnan(a)
    out = (rounded & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def trainable_mask():
    """(4, 64, 64) bool: rows the network uses (hidden unit 63 and head rows 40..63 are unused)."""
    m = np.zeros((LAYERS, WIDTH, WIDTH), dtype=bool)
    m[:3, :63, :] = True
    m[3, :OUT, :] = True
    return m


def encode(pos, normal, wo, box):
    """(n, 64) float64 features."""
    pos, normal, wo = (np.atleast_2d(np.asarray(v, dtype=np.float64)) for v in (pos, normal, wo))
    lo, hi = np.asarray(box[:3], np.float64), np.asarray(box[3:], np.float64)
    ext = hi - lo
    u = np.where(ext > 0, (pos - lo) / np.where(ext > 0, ext, 1.0), 0.5)
    u = np.clip(u, 0.0, 1.0)
    n = pos.shape[0]
    f = np.zeros((n, WIDTH))
    for k in range(5):
        s = u * (2.0 ** k)
        for a in range(3):
            f[:, 6 * k + 2 * a] = np.sin(np.pi * s[:, a])
            f[:, 6 * k + 2 * a + 1] = np.cos(np.pi * s[:, a])
    d = np.concatenate([normal, wo], axis=1)
    f[:, 30:36] = d
    for c in range(6):
        for k in range(2):
            s = d[:, c] * (2.0 ** k)
            f[:, 36 + 4 * c + 2 * k] = np.sin(np.pi * s)
            f[:, 36 + 4 * c + 2 * k + 1] = np.cos(np.pi * s)
    f[:, 63] = 1.0
    return f


def _weights(params, use_bf16):
    W = np.asarray(params, dtype=np.float64).reshape(LAYERS, WIDTH, WIDTH) * trainable_mask()
    return bf16(W) if use_bf16 else W


def forward(params, X0, use_bf16=True):
    """Returns (raw head outputs (n, 40), list of layer inputs X[0..3])."""
    W = _weights(params, use_bf16)
    X = bf16(X0) if use_bf16 else np.array(X0, dtype=np.float64)
    xs = [X]
    for l in range(LAYERS):
        Z = X @ W[l].T
        if l < 3:
            H = np.maximum(Z, 0.0)
            H[:, 63] = 1.0
            X = bf16(H) if use_bf16 else H
            xs.append(X)
        else:
            return Z[:, :OUT], xs


def lobes(raw):
    """(pi (n, 8), kappa (n, 8), mu (n, 8, 3), mu_len (n, 8)) from the raw head outputs."""
    raw = np.atleast_2d(raw)
    lg = raw[:, 0:8]
    e = np.exp(lg - lg.max(axis=1, keepdims=True))
    pi = e / e.sum(axis=1, keepdims=True)
    kappa = np.exp(np.clip(raw[:, 8:16], KAPPA_LOG_MIN, KAPPA_LOG_MAX))
    m = np.stack([raw[:, 16:24], raw[:, 24:32], raw[:, 32:40]], axis=2)
    ml = np.linalg.norm(m, axis=2)
    mu = m / np.maximum(ml, 1e-12)[..., None]
    return pi, kappa, mu, ml


def vmf_log_pdf(kappa, cos_mu):
    return np.log(kappa) - np.log(2 * np.pi) - np.log1p(-np.exp(-2 * kappa)) + kappa * (cos_mu - 1.0)


def log_q(raw, w):
    pi, kappa, mu, _ = lobes(raw)
    w = np.atleast_2d(w)
    cm = np.einsum("njk,nk->nj", mu, w)
    lf = np.log(np.maximum(pi, 1e-300)) + vmf_log_pdf(kappa, cm)
    mx = lf.max(axis=1, keepdims=True)
    return (mx + np.log(np.exp(lf - mx).sum(axis=1, keepdims=True)))[:, 0]


def mixture_pdf(raw, w):
    return np.exp(log_q(raw, w))


def head_grad(raw, w, weight, scale):
    """d(scale * -weight log q(w)) / d raw, shape (n, 40)."""
    pi, kappa, mu, ml = lobes(raw)
    w = np.atleast_2d(w)
    cm = np.einsum("njk,nk->nj", mu, w)
    lf = np.log(np.maximum(pi, 1e-300)) + vmf_log_pdf(kappa, cm)
    lq = log_q(raw, w)
    r = np.exp(lf - lq[:, None])
    c = (-np.asarray(weight, np.float64) * scale)[:, None]
    g = np.zeros((raw.shape[0], OUT))
    g[:, 0:8] = c * (r - pi)
    in_range = (raw[:, 8:16] > KAPPA_LOG_MIN) & (raw[:, 8:16] < KAPPA_LOG_MAX)
    dlogf_dk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (cm - 1.0)
    g[:, 8:16] = c * r * kappa * dlogf_dk * in_range
    dm = (w[:, None, :] - mu * cm[..., None]) * (c * r * kappa / np.maximum(ml, 1e-12))[..., None]
    g[:, 16:24], g[:, 24:32], g[:, 32:40] = dm[..., 0], dm[..., 1], dm[..., 2]
    return g


def loss_and_grad(params, records, box, scale=None, use_bf16=True):
    """records (n, 13): pos, normal, wo, wi, weight.  Returns (loss, grad (16384,))."""
    rec = np.asarray(records, dtype=np.float64)
    n = rec.shape[0]
    scale = 1.0 / n if scale is None else scale
    weight = np.where(np.isfinite(rec[:, 12]) & (rec[:, 12] >= 0), rec[:, 12], 0.0)
    X0 = encode(rec[:, 0:3], rec[:, 3:6], rec[:, 6:9], box)
    W = _weights(params, use_bf16)
    raw, xs = forward(params, X0, use_bf16)
    loss = float(np.sum(-weight * scale * log_q(raw, rec[:, 9:12])))
    G = np.zeros((n, WIDTH))
    G[:, :OUT] = head_grad(raw, rec[:, 9:12], weight, scale)
    if use_bf16:
        G = bf16(G)
    grad = np.zeros((LAYERS, WIDTH, WIDTH))
    for l in range(3, -1, -1):
        grad[l] = G.T @ xs[l]
        if l > 0:
            dX = G @ W[l]
            dX = dX * (xs[l] > 0)
            dX[:, 63] = 0.0
            G = bf16(dX) if use_bf16 else dX
    grad *= trainable_mask()
    return loss, grad.reshape(-1)


def loss_only(params, records, box, scale=None):
    """float64 loss without rounding (for finite differences)."""
    rec = np.asarray(records, dtype=np.float64)
    scale = 1.0 / rec.shape[0] if scale is None else scale
    X0 = encode(rec[:, 0:3], rec[:, 3:6], rec[:, 6:9], box)
    raw, _ = forward(params, X0, use_bf16=False)
    return float(np.sum(-rec[:, 12] * scale * log_q(raw, rec[:, 9:12])))


def init_params(seed):
    """Random parameters in the layout W[l][o][i] (unused rows zero), numpy RNG."""
    rng = np.random.default_rng(seed)
    W = np.zeros((LAYERS, WIDTH, WIDTH))
    for l in range(LAYERS):
        a = np.sqrt(6.0 / 64.0) * (1.0 if l < 3 else 0.5)
        W[l, :, :63] = rng.uniform(-a, a, size=(WIDTH, 63))
        W[l, :, 63] = rng.uniform(-0.1, 0.1, size=WIDTH)
    return (W * trainable_mask()).reshape(-1)


# ---------------------------------------------------------------- the reference's metallic bounce
def to_onb_ref(src, up, tangent):
    """to_onb of shared.wesl:39-46 as written: a combination of the cross-product vectors, which for
    an orthonormal frame equals -from_onb(src) rather than its inverse."""
    s = np.asarray(tangent, np.float64)
    up = np.asarray(up, np.float64)
    t = np.cross(up, s)
    return src[0] * np.cross(up, t) + src[1] * np.cross(t, s) + src[2] * np.cross(s, up)


def metal_frame(rd, n, tangent):
    """(V, R, axes): V = what get_normal hands sample_vndf_ggx (general.wesl:718); R = rd in the frame
    from_onb uses (tangent, normal, normal x tangent); axes = that frame's rows."""
    rd, n, tg = (np.asarray(x, np.float64) for x in (rd, n, tangent))
    axes = np.stack([tg, n, np.cross(n, tg)])
    return to_onb_ref(rd, n, tg), axes @ rd, axes


def metal_sample(V, R, ax, ay, u1, u2):
    """The reference's metallic bounce in from_onb's frame (y = the normal facing the ray):
    sample_vndf_ggx(seed, V) (general.wesl:1246-1281), reflect(rd, m) and, when that points below
    the surface, a mirror about the normal (:892-897).  u1, u2: (N,) uniforms; returns (N, 3)."""
    wi = np.array([V[0] * ax, V[1], V[2] * ay], np.float64)
    wi /= np.linalg.norm(wi)
    phi = 2.0 * np.pi * u1
    y = (1.0 - u2) * (1.0 + wi[1]) - wi[1]
    st = np.sqrt(np.clip(1.0 - y * y, 0.0, 1.0))
    c = np.stack([st * np.cos(phi), y, st * np.sin(phi)], 1) + wi
    m = np.stack([c[:, 0] * ax, c[:, 1], c[:, 2] * ay], 1)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    d = R[None, :] - 2.0 * (m @ R)[:, None] * m
    d[:, 1] = np.abs(d[:, 1])
    return d


def metal_pdf(V, R, ax, ay, w):
    """Density per solid angle of metal_sample's directions, derived independently of the CUDA code:
    the cap point p is uniform on {y >= -wi.y} (area 2 pi (1 + wi.y)); u = p + wi lies on the unit
    sphere through the origin, where a direction u has density 4 (u . wi) per unit area's worth of
    solid angle; m = normalize(S u) (S = diag(ax, 1, ay)) has Jacobian 1 / (ax ay |S^-1 m|^3); the
    reflection w = reflect(R, m) has Jacobian 1 / (4 |w . m|); the mirror adds the density of the
    mirrored direction.  w: (N, 3) unit directions in the same frame; 0 below the surface."""
    wi = np.array([V[0] * ax, V[1], V[2] * ay], np.float64)
    wi /= np.linalg.norm(wi)

    def raw(o):
        h = o - R[None, :]
        hl = np.linalg.norm(h, axis=1, keepdims=True)
        h = h / np.maximum(hl, 1e-300)
        h = np.where(h[:, 1:2] < 0, -h, h)
        us = h / np.array([ax, 1.0, ay])
        ul = np.linalg.norm(us, axis=1)
        u = us / ul[:, None]
        uw = u @ wi
        py = 2.0 * uw * u[:, 1] - wi[1]
        ok = (uw > 0) & (py >= -wi[1])
        dens = np.where(ok, 4.0 * uw / (2.0 * np.pi * (1.0 + wi[1])) / (ax * ay * ul ** 3), 0.0)
        wm = np.abs((o * h).sum(1))
        return np.where(wm > 0, dens / (4.0 * np.maximum(wm, 1e-300)), 0.0)

    w = np.asarray(w, np.float64).reshape(-1, 3)
    mirrored = w * np.array([1.0, -1.0, 1.0])
    return np.where(w[:, 1] > 0, raw(w) + raw(mirrored), 0.0)
