"""CPU restatement of the PSF surrogate network (TEST INFRASTRUCTURE ONLY).

The reference has no learned component; this module is the FP64 NumPy
definition of the network the GPU trains and evaluates, with the forward
pass and a hand-written backward pass, so the GPU's BF16 tensor-core forward
and gradients can be checked against it (and it against finite differences).

Network (per site; grid 64 x 64 = 4,096 pixels, width 32):

    h0  = X Wl^T + bl                                 lifting, X: (4096, 32)
    for l in 0..3:
        V   = F h_l                                   (576, 32): 288 modes, re/im rows
        Vo  = mix(V, R_l)                             per-mode complex 32x32 product
        z_l = h_l W_l^T + G Vo + b_l
        h_{l+1} = gelu(z_l)  (l < 3),  z_3 (l = 3)
    y   = h4 Wp^T + bp + base                         (4096, 16), planes 0..8 used

Modes: kx in {0..11, 52..63} (i.e. -12..-1), ky in 0..11, mode q = ikx*12 + iky,
theta_q(p) = 2 pi (kx x + ky y) / 64 for pixel p = 64 x + y.
F[2q] = cos theta, F[2q+1] = -sin theta (forward DFT rows, unnormalised);
G[p, 2q] = w_q cos theta, G[p, 2q+1] = -w_q sin theta with w_q = (1 if ky = 0
else 2) / 4096 (real part of the inverse transform).  F and G are rounded to
BF16 exactly as the GPU holds them.  Loss: mean over sites of
||y_s - t_s||^2 / ||t_s||^2 over planes 0..8.
"""

import numpy as np

GRID = 64
NPIX = GRID * GRID
WIDTH = 32
MODES = 12
NMODES = 2 * MODES * MODES       # 288 complex modes
NROWS = 2 * NMODES               # 576 real rows
PLANES = 9
OUT = 16                         # output channels (planes padded)
LAYERS = 4
GELU_C = np.sqrt(2.0 / np.pi)
GELU_A = 0.044715


def bf16_round(a):
    """Round float values to the nearest BF16 (ties to even), as float64."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def mode_table():
    kx = np.concatenate([np.arange(MODES), np.arange(GRID - MODES, GRID)])
    ky = np.arange(MODES)
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    return KX.reshape(-1), KY.reshape(-1)


def spectral_matrices():
    """(F (576, 4096), G (4096, 576)) rounded to BF16."""
    kx, ky = mode_table()
    x, y = np.divmod(np.arange(NPIX), GRID)
    th = 2 * np.pi * (np.outer(kx, x) + np.outer(ky, y)) / GRID     # (288, 4096)
    F = np.empty((NROWS, NPIX))
    F[0::2], F[1::2] = np.cos(th), -np.sin(th)
    w = np.where(ky == 0, 1.0, 2.0) / NPIX
    G = np.empty((NPIX, NROWS))
    G[:, 0::2], G[:, 1::2] = (w[:, None] * np.cos(th)).T, (-w[:, None] * np.sin(th)).T
    return bf16_round(F), bf16_round(G)


def init_params(seed=0, base=None):
    """Seeded initial parameters (FP64 arrays)."""
    rng = np.random.default_rng(seed)
    p = {"Wl": rng.normal(0, 1 / np.sqrt(18), (WIDTH, WIDTH)), "bl": np.zeros(WIDTH),
         "Wp": rng.normal(0, 1 / np.sqrt(WIDTH), (OUT, WIDTH)) * 1e-2, "bp": np.zeros(OUT)}
    p["Wl"][:, 18:] = 0.0
    p["Wp"][PLANES:] = 0.0
    for l in range(LAYERS):
        p[f"W{l}"] = rng.normal(0, 1 / np.sqrt(WIDTH), (WIDTH, WIDTH))
        p[f"b{l}"] = np.zeros(WIDTH)
        scale = 1.0 / (WIDTH * WIDTH)
        p[f"Rr{l}"] = rng.uniform(-scale, scale, (NMODES, WIDTH, WIDTH)) * NPIX / 64
        p[f"Ri{l}"] = rng.uniform(-scale, scale, (NMODES, WIDTH, WIDTH)) * NPIX / 64
    p["base"] = np.zeros((NPIX, OUT)) if base is None else np.asarray(base, float)
    return p


def gelu(z):
    return 0.5 * z * (1 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    u = GELU_C * (z + GELU_A * z ** 3)
    t = np.tanh(u)
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * GELU_C * (1 + 3 * GELU_A * z * z)


def _qmm(a, r):
    """(S, q, i) x (q, i, o) -> (S, q, o), batched over modes."""
    return np.matmul(a.transpose(1, 0, 2), r).transpose(1, 0, 2)


def _qmm_t(g, r):
    """(S, q, o) x (q, i, o)^T -> (S, q, i)."""
    return np.matmul(g.transpose(1, 0, 2), r.transpose(0, 2, 1)).transpose(1, 0, 2)


def _qouter(a, g):
    """sum over sites of a (S, q, i) outer g (S, q, o) -> (q, i, o)."""
    return np.matmul(a.transpose(1, 2, 0), g.transpose(1, 0, 2))


def mix(V, Rr, Ri):
    """V (S, 576, 32) -> Vo (S, 576, 32): per-mode complex V_q R_q."""
    vr, vi = V[:, 0::2], V[:, 1::2]                   # (S, 288, 32)
    out = np.empty_like(V)
    out[:, 0::2] = _qmm(vr, Rr) - _qmm(vi, Ri)
    out[:, 1::2] = _qmm(vr, Ri) + _qmm(vi, Rr)
    return out


def mix_backward(V, dVo, Rr, Ri):
    vr, vi = V[:, 0::2], V[:, 1::2]
    gr, gi = dVo[:, 0::2], dVo[:, 1::2]
    dV = np.empty_like(V)
    dV[:, 0::2] = _qmm_t(gr, Rr) + _qmm_t(gi, Ri)
    dV[:, 1::2] = -_qmm_t(gr, Ri) + _qmm_t(gi, Rr)
    dRr = _qouter(vr, gr) + _qouter(vi, gi)
    dRi = -_qouter(vi, gr) + _qouter(vr, gi)
    return dV, dRr, dRi


def forward(p, X, mats=None):
    """X (S, 4096, 32) -> prediction (S, 4096, 16) and the cache for backward."""
    F, G = spectral_matrices() if mats is None else mats
    h = X @ p["Wl"].T + p["bl"]
    cache = {"X": X, "h": [h], "z": [], "V": []}
    for l in range(LAYERS):
        V = np.matmul(F, h)
        Vo = mix(V, p[f"Rr{l}"], p[f"Ri{l}"])
        z = h @ p[f"W{l}"].T + np.matmul(G, Vo) + p[f"b{l}"]
        cache["V"].append(V)
        cache["z"].append(z)
        h = gelu(z) if l < LAYERS - 1 else z
        cache["h"].append(h)
    y = h @ p["Wp"].T + p["bp"] + p["base"]
    return y, cache


def loss(y, T):
    """Mean over sites of the squared relative L2 error over planes 0..8."""
    d = (y - T)[..., :PLANES]
    num = (d ** 2).sum((1, 2))
    den = (T[..., :PLANES] ** 2).sum((1, 2))
    return float((num / den).mean())


def backward(p, cache, y, T, mats=None):
    """Gradients of ``loss`` with respect to every trained parameter."""
    F, G = spectral_matrices() if mats is None else mats
    S = y.shape[0]
    den = (T[..., :PLANES] ** 2).sum((1, 2))
    dy = np.zeros_like(y)
    dy[..., :PLANES] = 2 * (y - T)[..., :PLANES] / (S * den[:, None, None])
    g = {}
    h4 = cache["h"][LAYERS]
    g["Wp"] = np.einsum("spk,spi->ki", dy, h4)
    g["bp"] = dy.sum((0, 1))
    dh = dy @ p["Wp"]
    for l in reversed(range(LAYERS)):
        z = cache["z"][l]
        dz = dh * gelu_grad(z) if l < LAYERS - 1 else dh
        h = cache["h"][l]
        g[f"W{l}"] = np.einsum("spo,spi->oi", dz, h)
        g[f"b{l}"] = dz.sum((0, 1))
        dVo = np.matmul(G.T, dz)
        dV, g[f"Rr{l}"], g[f"Ri{l}"] = mix_backward(cache["V"][l], dVo, p[f"Rr{l}"], p[f"Ri{l}"])
        dh = dz @ p[f"W{l}"] + np.matmul(F.T, dV)
    g["Wl"] = np.einsum("spo,spc->oc", dh, cache["X"])
    g["bl"] = dh.sum((0, 1))
    return g
