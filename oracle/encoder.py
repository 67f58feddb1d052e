"""CPU restatement (numpy, float64) of the sequence encoder of the learned-proposal path: forward
pass, pair loss and hand-derived backward pass.  Test infrastructure only: the tests check the
CUDA training kernels' loss and gradients against this, and this against finite differences.

The model (no counterpart in the reference; the architecture is the one the proposal path is
specified with: 2 conv layers + 2 attention layers, width 128, 64-d output, one-hot input padded
to length 32):

    one-hot codes x[t] (t < L <= 32, alphabet 24)
    h1[t] = relu(b1 + sum_{o in -1,0,1} W1[o][x[t+o]])            conv k=3, 24 -> 128
    h2[t] = h1[t] + relu(b2 + [h1[t-1], h1[t], h1[t+1]] @ W2)     conv k=3, 128 -> 128 (+ skip)
    for each of 2 attention layers (single head, d = 128):
        qkv = h @ Wqkv + bqkv;  q, k, v = split(qkv)
        a[t] = softmax_u<L(q[t] . k[u] / sqrt(128));  o[t] = sum_u a[t][u] v[u]
        h = h + o @ Wo + bo
    p = mean_{t<L} h[t];  e = p @ Wout + bout;  z = e / |e|        (64-d, unit length)

Pair loss over pairs (z_a, z_b) with exact gap-block score s:
    d = |z_a - z_b|^2,  target = min(s, CLIP) / (CLIP / 2),  loss = mean (d - target)^2
so a distance of 0 means identical and 2 (orthogonal) means a score at or beyond CLIP.
"""
from __future__ import annotations

import numpy as np

A = 24        # amino-acid codes
W = 128       # width
E = 64        # embedding size
P = 32        # padded length
CLIP = 64.0   # scores at or above this are "far"

# parameter blocks in order: (name, shape)
SHAPES = [("W1", (3, A, W)), ("b1", (W,)), ("W2", (3 * W, W)), ("b2", (W,)),
          ("Wqkv0", (W, 3 * W)), ("bqkv0", (3 * W,)), ("Wo0", (W, W)), ("bo0", (W,)),
          ("Wqkv1", (W, 3 * W)), ("bqkv1", (3 * W,)), ("Wo1", (W, W)), ("bo1", (W,)),
          ("Wout", (W, E)), ("bout", (E,))]


def param_count() -> int:
    return int(sum(np.prod(s) for _, s in SHAPES))


def unpack(flat: np.ndarray) -> dict[str, np.ndarray]:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def pack(params: dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([np.asarray(params[n], np.float64).ravel() for n, _ in SHAPES])


def init_params(seed: int) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (a reproducible start; the
    CUDA encoder is initialised from the same array)."""
    rng = np.random.default_rng(seed)
    fan = {"W1": 3, "W2": 3 * W, "Wqkv0": W, "Wo0": W, "Wqkv1": W, "Wo1": W, "Wout": W}
    parts = []
    for name, shape in SHAPES:
        if name in fan:
            lim = 1.0 / np.sqrt(fan[name])
            parts.append(rng.uniform(-lim, lim, size=shape).ravel())
        else:
            parts.append(np.zeros(int(np.prod(shape))))
    return np.concatenate(parts).astype(np.float32)


def _shift(h, lens, o):
    """h[t+o] with zeros outside [0, L)."""
    S = h.shape[0]
    out = np.zeros_like(h)
    t = np.arange(P)
    for s in range(S):
        src = t + o
        ok = (src >= 0) & (src < lens[s]) & (t < lens[s])
        out[s, t[ok]] = h[s, src[ok]]
    return out


def forward(flat, codes, lens, keep=False):
    """codes uint8 [S, P], lens [S] -> z [S, E] (and the activations when keep)."""
    p = unpack(np.asarray(flat, np.float64))
    S = codes.shape[0]
    mask = (np.arange(P)[None, :] < lens[:, None]).astype(np.float64)[..., None]  # [S,P,1]
    pre1 = np.zeros((S, P, W)) + p["b1"]
    for oi, o in enumerate((-1, 0, 1)):
        t = np.arange(P)
        for s in range(S):
            src = t + o
            ok = (src >= 0) & (src < lens[s]) & (t < lens[s])
            pre1[s, t[ok]] += p["W1"][oi][codes[s, src[ok]]]
    h1 = np.maximum(pre1, 0) * mask
    x2 = np.concatenate([_shift(h1, lens, -1), h1, _shift(h1, lens, 1)], axis=2)  # [S,P,384]
    pre2 = x2 @ p["W2"] + p["b2"]
    h = (h1 + np.maximum(pre2, 0)) * mask
    acts = {"mask": mask, "pre1": pre1, "h1": h1, "x2": x2, "pre2": pre2, "att": []}
    keymask = np.where(np.arange(P)[None, None, :] < lens[:, None, None], 0.0, -np.inf)
    for l in range(2):
        qkv = h @ p[f"Wqkv{l}"] + p[f"bqkv{l}"]
        q, k, v = qkv[..., :W], qkv[..., W:2 * W], qkv[..., 2 * W:]
        sc = q @ k.transpose(0, 2, 1) / np.sqrt(W) + keymask
        sc = sc - sc.max(axis=2, keepdims=True)
        a = np.exp(sc)
        a /= a.sum(axis=2, keepdims=True)
        a = a * mask  # padded query rows carry nothing
        o = a @ v
        hn = (h + o @ p[f"Wo{l}"] + p[f"bo{l}"]) * mask
        acts["att"].append({"h": h, "q": q, "k": k, "v": v, "a": a, "o": o})
        h = hn
    pool = h.sum(axis=1) / lens[:, None]
    e = pool @ p["Wout"] + p["bout"]
    n = np.linalg.norm(e, axis=1, keepdims=True)
    z = e / n
    acts.update(h=h, pool=pool, e=e, n=n)
    return (z, acts) if keep else z


def pair_loss(z, scores):
    """Loss over consecutive pairs (z[2i], z[2i+1]) and dL/dz."""
    za, zb = z[0::2], z[1::2]
    d = ((za - zb) ** 2).sum(axis=1)
    tgt = np.minimum(np.asarray(scores, np.float64), CLIP) / (CLIP / 2)
    r = d - tgt
    loss = float((r ** 2).mean())
    g = 2 * r / len(r)                       # dL/dd
    dz = np.zeros_like(z)
    dz[0::2] = (2 * g)[:, None] * (za - zb)
    dz[1::2] = -(2 * g)[:, None] * (za - zb)
    return loss, dz


def backward(flat, codes, lens, scores):
    """(loss, gradient of the mean pair loss w.r.t. the flat parameters)."""
    p = unpack(np.asarray(flat, np.float64))
    z, ac = forward(flat, codes, lens, keep=True)
    loss, dz = pair_loss(z, scores)
    S = codes.shape[0]
    g = {name: np.zeros(shape) for name, shape in SHAPES}
    mask = ac["mask"]
    # z = e / n
    e, n = ac["e"], ac["n"]
    de = dz / n - e * ((dz * e).sum(axis=1, keepdims=True) / n ** 3)
    g["Wout"] = ac["pool"].T @ de
    g["bout"] = de.sum(axis=0)
    dpool = de @ p["Wout"].T
    dh = np.repeat((dpool / lens[:, None])[:, None, :], P, axis=1) * mask
    for l in (1, 0):
        at = ac["att"][l]
        # h_next = (h + o Wo + bo) * mask
        g[f"Wo{l}"] = np.einsum("spi,spj->ij", at["o"], dh)
        g[f"bo{l}"] = dh.sum(axis=(0, 1))
        do = dh @ p[f"Wo{l}"].T
        dhp = dh.copy()
        # o = a v
        da = do @ at["v"].transpose(0, 2, 1)
        dv = at["a"].transpose(0, 2, 1) @ do
        # softmax rows (padded rows have a = 0 and contribute nothing)
        ds = at["a"] * (da - (da * at["a"]).sum(axis=2, keepdims=True))
        ds /= np.sqrt(W)
        dq = ds @ at["k"]
        dk = ds.transpose(0, 2, 1) @ at["q"]
        dqkv = np.concatenate([dq, dk, dv], axis=2)
        g[f"Wqkv{l}"] = np.einsum("spi,spj->ij", at["h"], dqkv)
        g[f"bqkv{l}"] = dqkv.sum(axis=(0, 1))
        dh = (dhp + dqkv @ p[f"Wqkv{l}"].T) * mask
    # h = (h1 + relu(pre2)) * mask
    dpre2 = dh * (ac["pre2"] > 0)
    g["W2"] = np.einsum("spi,spj->ij", ac["x2"], dpre2)
    g["b2"] = dpre2.sum(axis=(0, 1))
    dx2 = dpre2 @ p["W2"].T
    dh1 = dh + dx2[..., W:2 * W] + _shift(dx2[..., :W], lens, 1) + _shift(dx2[..., 2 * W:], lens, -1)
    dh1 *= mask
    dpre1 = dh1 * (ac["pre1"] > 0)
    g["b1"] = dpre1.sum(axis=(0, 1))
    for oi, o in enumerate((-1, 0, 1)):
        t = np.arange(P)
        for s in range(S):
            src = t + o
            ok = (src >= 0) & (src < lens[s]) & (t < lens[s])
            np.add.at(g["W1"][oi], codes[s, src[ok]], dpre1[s, t[ok]])
    return loss, pack(g)


def loss_only(flat, codes, lens, scores) -> float:
    return pair_loss(forward(flat, codes, lens), scores)[0]
