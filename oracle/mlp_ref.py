"""CPU reference of the 4-64-64-1 temperature-guess MLP (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: the checker for the GPU training kernels.  FP64 arithmetic; with
bf16=True the same operands are rounded to bfloat16 where the GPU feeds the tensor cores
(hidden activations H1, the 64x64 weights W2 and the hidden-layer gradient dH2), so the two
agree to FP32 accumulation error.  Parameter layout: W1[64][4], b1[64], W2[64][64] (out, in),
b2[64], W3[64], b3.
"""
import numpy as np

NPARAM = 4545
OUT_SCALE, OUT_SHIFT = 0.5, -0.75   # log10 T = prior(X) + OUT_SCALE * y + OUT_SHIFT
LOG10_1P5_RGAS = 8.095925           # log10(3/2 R), R = 8.31446261815324e7 erg/(g K)
MINUS_LOG10_ARAD = 14.121147        # -log10(a), a = 7.565767381646406e-15 erg/(cm^3 K^4)


def bf16(a):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[0:256].reshape(64, 4), p[256:320], p[320:4416].reshape(64, 64), p[4416:4480], p[4480:4544], p[4544])


def forward(p, X, use_bf16=True):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    H1 = np.maximum(X @ W1.T + b1, 0.0)
    H1b = bf16(H1) if use_bf16 else H1
    W2b = bf16(W2) if use_bf16 else W2
    H2 = np.maximum(H1b @ W2b.T + b2, 0.0)
    y = H2 @ W3 + b3
    return y, (H1, H1b, W2b, H2)


def loss_and_grad(p, X, t, use_bf16=True):
    """Mean squared loss and its gradient with respect to all parameters."""
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    B = X.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(p)
    y, (H1, H1b, W2b, H2) = forward(p, X, use_bf16)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / B
    g_W3 = H2.T @ dy
    g_b3 = dy.sum()
    dH2 = np.outer(dy, W3) * (H2 > 0)
    g_b2 = dH2.sum(axis=0)
    dH2b = bf16(dH2) if use_bf16 else dH2
    g_W2 = dH2b.T @ H1b
    dH1 = (dH2b @ W2b) * (H1 > 0)
    g_W1 = dH1.T @ X
    g_b1 = dH1.sum(axis=0)
    g = np.concatenate([g_W1.ravel(), g_b1, g_W2.ravel(), g_b2, g_W3, [g_b3]])
    return loss, g


def features(rho, e_th, abar, zbar):
    """Normalised inputs: log10 rho, log10 of the thermal energy e - E(rho, T_lo), Abar, Zbar."""
    return np.stack([(np.log10(rho) - 3.5) / 5.5, (np.log10(np.maximum(e_th, 1e-300)) - 19.5) / 8.5,
                     (abar - 28.5) / 27.5, (zbar - 14.0) / 14.0], axis=-1).astype(np.float32)


def prior(X):
    """log10 T that ideal ions plus radiation alone would need to hold the thermal energy."""
    X = np.asarray(X, dtype=np.float64)
    lrho = 5.5 * X[:, 0] + 3.5
    le = 8.5 * X[:, 1] + 19.5
    abar = 27.5 * X[:, 2] + 28.5
    l_ion = le + np.log10(abar) - LOG10_1P5_RGAS
    l_rad = 0.25 * (le + lrho + MINUS_LOG10_ARAD)
    return np.minimum(l_ion, l_rad) - 0.25 * np.log10(1.0 + 10.0 ** (-4.0 * np.abs(l_ion - l_rad)))


def guess_log10T(p, X, use_bf16=True):
    """The learned guess log10 T for normalised inputs X (n x 4)."""
    y, _ = forward(p, np.asarray(X, dtype=np.float64), use_bf16)
    return prior(X) + OUT_SCALE * y + OUT_SHIFT
