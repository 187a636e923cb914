"""numpy restatement of the learned troubled-cell indicator's features and
forward pass (the layout of include/kfvm_b200.h), used by the tests as the
checker of the CUDA kernels.  Patches read the halo through the periodic wrap or
the outflow mirror, as the halo fill does."""
import numpy as np

R = 2
NH = 32


def bf16_to_f32(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def f32_to_bf16(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = u + 0x7FFF + ((u >> 16) & 1)
    return (u >> 16).astype(np.uint16)


def pressure(u, gamma, glm=False):
    rho = u[0]
    ke = 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / rho
    eint = u[4] - ke
    if glm:
        eint = eint - 0.5 * (u[5] ** 2 + u[6] ** 2 + u[7] ** 2) - 0.5 * u[8] ** 2
    return (gamma - 1.0) * eint


def features(state, cfg, cells):
    """Features of the given cells from an interior state (nv, n): density and
    pressure in float64 rounded to float32, differences, maxima, scales and
    products in float32 (the kernels' definition)."""
    dim = cfg.dim
    nz = cfg.nz if dim == 3 else 1
    shape = (nz, cfg.ny, cfg.nx)
    nv = state.shape[0]
    u = state.reshape((nv,) + shape)
    rho = u[0]
    p = pressure(u, cfg.gamma, glm=(nv == 9))
    modes = []
    for ax, (lo, hi) in ((2, (0, 1)), (1, (2, 3)), (0, (4, 5))):
        if dim == 2 and ax == 0:
            modes.append(None)
            continue
        modes.append("wrap" if cfg.bc[lo] == 0 else "symmetric")

    def pad(a):
        for ax, m in zip((2, 1, 0), modes):
            if m is None:
                continue
            w = [(0, 0)] * 3
            w[ax] = (R, R)
            a = np.pad(a, w, mode=m)
        return a
    # density and pressure in FP64, rounded to FP32; the rest in FP32
    rp, pp = pad(rho).astype(np.float32), pad(p).astype(np.float32)
    zr = R if dim == 3 else 0
    out = np.empty((len(cells), 2 * (2 * R + 1) ** dim), dtype=np.float32)
    f4 = np.float32(1e-4)
    tiny = np.float32(1e-30)
    for n, c in enumerate(cells):
        k, rem = divmod(int(c), cfg.nx * cfg.ny)
        j, i = divmod(rem, cfg.nx)
        kk = k + zr
        sl = (slice(kk - zr, kk + zr + 1), slice(j, j + 2 * R + 1), slice(i, i + 2 * R + 1))
        pr, pq = rp[sl].ravel(), pp[sl].ravel()
        rc, pc = rp[kk, j + R, i + R], pp[kk, j + R, i + R]
        dr, dq = pr - rc, pq - pc
        sr = np.float32(1.0) / (np.abs(dr).max() + f4 * np.abs(rc) + tiny)
        sq = np.float32(1.0) / (np.abs(dq).max() + f4 * np.abs(pc) + tiny)
        out[n] = np.concatenate([dr * sr, dq * sq])
    return out


def unpack(w_bf16, ni):
    w = bf16_to_f32(w_bf16).astype(np.float64)
    o = 0
    W1 = w[o:o + NH * ni].reshape(NH, ni); o += NH * ni
    b1 = w[o:o + NH]; o += NH
    W2 = w[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = w[o:o + NH]; o += NH
    w3 = w[o:o + NH]; o += NH
    b3 = w[o]
    return W1, b1, W2, b2, w3, b3


def gelu(x):
    """GELU in its tanh approximation, x sigma(2 sqrt(2/pi) (x + 0.044715 x^3))."""
    c0 = 2.0 * np.sqrt(2.0 / np.pi)
    return x / (1.0 + np.exp(-x * (c0 + c0 * 0.044715 * x * x)))


def probability(w_bf16, x):
    """Forward pass in float64 with the BF16 weights: x (m, NI) -> (m,)."""
    x = np.asarray(x, dtype=np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(w_bf16, x.shape[1])
    h1 = gelu(x @ W1.T + b1)
    h2 = gelu(h1 @ W2.T + b2)
    z = h2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z))
