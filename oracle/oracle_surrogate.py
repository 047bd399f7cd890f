"""CPU oracle of the scatter surrogate's network (test infrastructure only).

Restates, in numpy, the coordinate MLP that the library trains on the tensor
cores (gpu-spect-pet-sysmat_b200/csrc/surrogate_net.cu):

    rho(d, v) = g(d) . h(v)
    h(v) = trunk over Fourier features of the voxel centre: for each axis with
           n voxels, c = 2 (i + 0.5) / n - 1 and w_j = pi/2 min(n/2, 8)^(j / (F - 1)),
           features (sin w_j c, cos w_j c) for j < F (axis-major); `layers`
           linear layers of `width`, SiLU between them, the last one linear;
    g(d) = P e_d + b_P.

Loss of a batch: sum_{d, j} wgt[d][col_j] (rho(d, vox_j) - rho_t[d][col_j])^2 / (N B),
and its gradient with respect to the parameter vector (for l < layers: W_l
[width][in_l], b_l [width]; then E [N][emb], P [width][emb], b_P [width]; each
block starting at a multiple of 64 floats).

With ``bf16=True`` the oracle rounds to bfloat16 exactly where the GPU path
does (GEMM operands: features, weights, activations, G, the output gradient
and the backward operands), so the comparison isolates the arithmetic; with
``bf16=False`` it is the plain fp64 model, whose gradient is pinned by
finite differences in tests/test_surrogate_oracle.py.  The network has no
counterpart in the reference project: it is the learned part of the scatter
surrogate that the project adds around the reference's exact scatter kernel.
"""
import numpy as np


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(a)
    if nan.any():
        out[nan] = np.nan
    return out


def layout(n_crystals, layers, width, freqs, emb):
    """Offsets and shapes of the parameter blocks."""
    shapes = []
    for l in range(layers):
        fin = 6 * freqs if l == 0 else width
        shapes += [(width, fin), (width,)]
    shapes += [(n_crystals, emb), (width, emb), (width,)]
    offs, at = [], 0
    for s in shapes:
        offs.append(at)
        at += (int(np.prod(s)) + 63) // 64 * 64
    return offs, shapes, at


def unpack(params, offs, shapes):
    p = np.asarray(params, dtype=np.float64)
    return [p[o:o + int(np.prod(s))].reshape(s) for o, s in zip(offs, shapes)]


def fourier(vox, grid, freqs, round_bf16=True):
    nx, ny, nz = grid
    vox = np.asarray(vox, dtype=np.int64)
    idx = (vox % nx, (vox // nx) % ny, vox // (nx * ny))
    cols = []
    for axis, n in enumerate((nx, ny, nz)):
        c = (2.0 * (idx[axis].astype(np.float32) + np.float32(0.5)) / np.float32(n) - np.float32(1.0)).astype(np.float32)
        j = np.arange(freqs, dtype=np.float32)
        e = j / np.float32(freqs - 1) if freqs > 1 else np.zeros(1, np.float32)
        w = np.float32(1.57079632679489662) * np.power(np.float32(min(0.5 * n, 8.0)), e).astype(np.float32)
        a = (c[:, None] * w[None, :]).astype(np.float32).astype(np.float64)   # the product rounds to fp32
        feats = np.empty((vox.size, 2 * freqs))
        feats[:, 0::2] = np.sin(a)
        feats[:, 1::2] = np.cos(a)
        cols.append(feats)
    x = np.concatenate(cols, axis=1)
    return bf16(x) if round_bf16 else x


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _r(x, on):
    return bf16(x) if on else np.asarray(x, dtype=np.float64)


def forward(params, offs, shapes, grid, freqs, vox, round_bf16=True):
    """rho[d][j] for voxels vox (N x len(vox)) and the intermediate values."""
    blocks = unpack(params, offs, shapes)
    L = (len(blocks) - 3) // 2
    Ws, bs = blocks[0:2 * L:2], blocks[1:2 * L:2]
    E, P, bP = blocks[2 * L:]
    x = fourier(vox, grid, freqs, round_bf16)
    ins, zs = [], []
    a = x
    for l in range(L):
        ins.append(a)
        z = a @ _r(Ws[l], round_bf16).T + bs[l]
        zs.append(z)
        a = _r(_silu(z), round_bf16) if l + 1 < L else _r(z, round_bf16)
    H = a
    G = _r(E, round_bf16) @ _r(P, round_bf16).T + bP
    Gb = _r(G, round_bf16)
    return Gb @ H.T, dict(ins=ins, zs=zs, H=H, G=G, Gb=Gb, Ws=Ws, E=E, P=P, L=L)


def loss_grad(params, offs, shapes, grid, freqs, vox, col, rho, wgt, round_bf16=True):
    """Loss and gradient vector (float64) of one batch."""
    yhat, c = forward(params, offs, shapes, grid, freqs, vox, round_bf16)
    N, B = yhat.shape
    col = np.asarray(col, dtype=np.int64)
    rt = np.asarray(rho, dtype=np.float64)[:, col]
    wt = np.asarray(wgt, dtype=np.float64)[:, col]
    r = yhat - rt
    loss = float((wt * r * r).sum() / (N * B))
    dy = _r(2.0 * wt * r / (N * B), round_bf16)
    grads = [None] * len(shapes)
    L = c["L"]
    dG = dy @ c["H"]
    dz = dy.T @ c["Gb"]
    dGb = _r(dG, round_bf16)
    grads[2 * L + 1] = dGb.T @ _r(c["E"], round_bf16)
    grads[2 * L + 2] = dG.sum(axis=0)
    grads[2 * L] = dGb @ _r(c["P"], round_bf16)
    for l in range(L - 1, -1, -1):
        dzb = _r(dz, round_bf16)
        grads[2 * l] = dzb.T @ c["ins"][l]
        grads[2 * l + 1] = dz.sum(axis=0)
        if l > 0:
            da = dzb @ _r(c["Ws"][l], round_bf16)
            z = c["zs"][l - 1]
            s = 1.0 / (1.0 + np.exp(-z))
            dz = da * s * (1.0 + z * (1.0 - s))
    g = np.zeros(len(params))
    for o, s, v in zip(offs, shapes, grads):
        g[o:o + int(np.prod(s))] = np.asarray(v).reshape(-1)
    return loss, g


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1); returns new (w, m, v)."""
    m = b1 * m + (1.0 - b1) * g
    v = b2 * v + (1.0 - b2) * g * g
    w = w - lr * (m / (1.0 - b1 ** step)) / (np.sqrt(v / (1.0 - b2 ** step)) + eps)
    return w, m, v


def init_params(n_crystals, layers, width, freqs, emb, seed=0):
    """Random parameters for checks (not the library's initialisation)."""
    rng = np.random.default_rng(seed)
    offs, shapes, n = layout(n_crystals, layers, width, freqs, emb)
    p = np.zeros(n, dtype=np.float32)
    for i, (o, s) in enumerate(zip(offs, shapes)):
        fan = s[1] if len(s) == 2 else 1
        p[o:o + int(np.prod(s))] = (rng.uniform(-1, 1, int(np.prod(s))) / np.sqrt(fan)).astype(np.float32)
    return p, offs, shapes
