"""CPU oracle of the learned proposal (test infrastructure only; never part of the product path).

The learned proposal has no counterpart in the reference; this file restates, in numpy, what
the engine's kernels compute so the GPU path can be checked:
  * the network 64 -> 128 -> 128 -> 16 with the kernels' rounding points: features, weights and
    hidden activations in BF16 (round to nearest even), products accumulated exactly here
    (float64) where the tensor cores accumulate in FP32, biases in FP32;
  * its gradients for the mean masked cross-entropy, with the backward operands rounded to BF16
    where the kernels feed them to the tensor cores, and the bias gradients from the unrounded
    FP32 values (rounding=False gives the exact float64 gradient of the same network);
  * the features of a vertex (candidate slots = 14 neighbour blocks with the most edges to the
    vertex, ties to the lower block id; block degree d_out + d_in; BF16 values);
  * q(s | v) of the mixture (1 - eps) softmax + eps uniform, the draw, and the reverse-state
    features.
Block degrees and the neighbour lists follow the engine's conventions, which are those of
the reference: the out list keeps the self loop, the in list drops it, d_in counts it
(src/finetune.cpp:491-492, src/blockmodel/blockmodel.cpp:187-255).
"""
import numpy as np

IN, HID, OUT, SLOTS, ESCAPE = 64, 128, 16, 14, 14
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
PARAMS = OFF_B3 + OUT


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p)
    if p.dtype != np.float64:
        p = p.astype(np.float32)
    return (p[OFF_W1:OFF_B1].reshape(HID, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(OUT, HID), p[OFF_B3:])


def _mm(a, b):
    return np.asarray(a, np.float64) @ np.asarray(b, np.float64)


def _rounders(rounding):
    """(BF16 rounding, FP32 cast) of the kernels, or the identity in float64 (rounding=False)."""
    if rounding:
        return bf16, (lambda a: np.asarray(a, np.float32))
    ident = (lambda a: np.asarray(a, np.float64))
    return ident, ident


def forward(params, X, keep=False, rounding=True):
    """logits[n][16]; rounding=False evaluates the same network exactly in float64."""
    R, F = _rounders(rounding)
    W1, b1, W2, b2, W3, b3 = unpack(params)
    Xb = R(X)
    h1 = R(np.maximum(F(_mm(Xb, R(W1).T)) + b1, 0.0))
    h2 = R(np.maximum(F(_mm(h1, R(W2).T)) + b2, 0.0))
    logits = F(_mm(h2, R(W3).T)) + b3
    if keep:
        return logits, (Xb, h1, h2)
    return logits


def mask(nvalid):
    j = np.arange(OUT)[None, :]
    nv = np.asarray(nvalid)[:, None]
    return ((j < SLOTS) & (j < nv)) | (j == ESCAPE)


def loss_of(params, X, target, nvalid, rounding=True):
    """Mean masked cross-entropy over the rows with target >= 0."""
    logits = forward(params, X, rounding=rounding)
    t = np.asarray(target)
    on = t >= 0
    L = np.where(mask(nvalid), np.asarray(logits, np.float64), -np.inf)
    mx = L.max(axis=1, keepdims=True)
    lse = mx[:, 0] + np.log(np.exp(L - mx).sum(axis=1))
    rows = np.arange(len(t))[on]
    return float((lse[on] - L[rows, t[on]]).sum() / max(int(on.sum()), 1))


def gradients(params, X, target, nvalid, rounding=True):
    """Gradient vector (PARAMS, float64) and mean loss over rows with target >= 0."""
    R, F = _rounders(rounding)
    W1, b1, W2, b2, W3, b3 = unpack(params)
    logits, (Xb, h1, h2) = forward(params, X, keep=True, rounding=rounding)
    t = np.asarray(target)
    m = mask(nvalid)
    on = t >= 0
    count = max(int(on.sum()), 1)
    L = np.where(m, np.asarray(logits, np.float64), -np.inf)
    mx = L.max(axis=1, keepdims=True)
    e = np.where(m, np.exp(L - mx), 0.0)
    S = e.sum(axis=1, keepdims=True)
    p = e / S
    onehot = np.zeros_like(p)
    onehot[np.arange(len(t))[on], t[on]] = 1.0
    dz3 = F(np.where(on[:, None], (p - onehot) / count, 0.0))
    loss = -(np.log(p[np.arange(len(t))[on], t[on]])).sum() / count
    dz3b = R(dz3)
    gW3 = _mm(dz3b.T, h2)
    gb3 = np.asarray(dz3, np.float64).sum(0)
    dh2 = F(_mm(dz3b, R(W3)))
    dz2 = F(np.where(h2 > 0, dh2, 0.0))
    dz2b = R(dz2)
    gW2 = _mm(dz2b.T, h1)
    gb2 = np.asarray(dz2, np.float64).sum(0)
    dh1 = F(_mm(dz2b, R(W2)))
    dz1 = F(np.where(h1 > 0, dh1, 0.0))
    dz1b = R(dz1)
    gW1 = _mm(dz1b.T, Xb)
    gb1 = np.asarray(dz1, np.float64).sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]).astype(np.float64)
    return g, float(loss)


def _f32(x):
    return np.float32(x)


def feat_degree(dtot, inv_log2E):
    return _f32(np.log1p(_f32(dtot))) * _f32(inv_log2E)


def inv_log2E(E):
    return _f32(1.0 / np.log1p(2.0 * max(E, 1)))


class Graph:
    """Out / in neighbour lists with the engine's conventions, from an edge list (deduplicated)."""

    def __init__(self, V, src, dst):
        seen = set()
        self.V = V
        self.out = [[] for _ in range(V)]
        self.inn = [[] for _ in range(V)]
        self.self = np.zeros(V, np.int32)
        for a, b in zip(np.asarray(src).tolist(), np.asarray(dst).tolist()):
            if (a, b) in seen:
                continue
            seen.add((a, b))
            self.out[a].append(b)
            if a == b:
                self.self[a] = 1
            else:
                self.inn[b].append(a)
        self.E = len(seen)


def block_degrees(g, b, B):
    d_out = np.zeros(B, np.int64)
    d_in = np.zeros(B, np.int64)
    for v in range(g.V):
        d_out[b[v]] += len(g.out[v])
        d_in[b[v]] += len(g.inn[v]) + g.self[v]
    return d_out, d_in


def global_features(k_out, k_in, B, nvalid, c_cur, kf, self, dtot_cur, inv):
    return np.array([_f32(np.log1p(_f32(k_out))) / _f32(5), _f32(np.log1p(_f32(k_in))) / _f32(5),
                     _f32(np.log(_f32(B))) / _f32(10), _f32(nvalid) / _f32(14), _f32(c_cur) / kf,
                     1.0 if self else 0.0, feat_degree(dtot_cur, inv), 1.0], np.float32)


def vertex_features(g, b, B, d_out, d_in, v):
    """(features[64] as BF16 values in float32, slots [(block, cout, cin)], r, k_out, k_in, self)."""
    r = int(b[v])
    cout, cin = {}, {}
    for u in g.out[v]:
        if u != v:
            cout[b[u]] = cout.get(b[u], 0) + 1
    for u in g.inn[v]:
        cin[b[u]] = cin.get(b[u], 0) + 1
    blocks = set(cout) | set(cin)
    cand = sorted(blocks, key=lambda x: (-(cout.get(x, 0) + cin.get(x, 0)), x))[:SLOTS]
    k_out, k_in, self = len(g.out[v]), len(g.inn[v]), int(g.self[v])
    k = k_out + k_in
    kf = _f32(k if k > 0 else 1)
    inv = inv_log2E(g.E)
    f = np.zeros(IN, np.float32)
    slots = []
    c_r = 0
    for j, u in enumerate(cand):
        co, ci = cout.get(u, 0), cin.get(u, 0)
        slots.append((int(u), co, ci))
        f[4 * j] = _f32(co) / kf
        f[4 * j + 1] = _f32(ci) / kf
        f[4 * j + 2] = feat_degree(d_out[u] + d_in[u], inv)
        f[4 * j + 3] = 1.0 if u == r else 0.0
        if u == r:
            c_r = co + ci
    f[56:64] = global_features(k_out, k_in, B, len(cand), c_r, kf, self, d_out[r] + d_in[r], inv)
    return bf16(f), slots, r, k_out, k_in, self


def reverse_features(F1, slots, r, s, k_out, k_in, self, B, d_out, d_in, E):
    """Features of the vertex after moving it from r to s, from the current state."""
    f = np.array(F1, np.float32).copy()
    inv = inv_log2E(E)
    mv = k_out + k_in + self
    dt_r = int(d_out[r] + d_in[r]) - mv
    dt_s = int(d_out[s] + d_in[s]) + mv
    c_s = 0
    for j, (u, co, ci) in enumerate(slots):
        if u == r:
            f[4 * j + 2] = feat_degree(dt_r, inv)
            f[4 * j + 3] = 0.0
        if u == s:
            f[4 * j + 2] = feat_degree(dt_s, inv)
            f[4 * j + 3] = 1.0
            c_s = co + ci
    k = k_out + k_in
    kf = _f32(k if k > 0 else 1)
    gl = global_features(k_out, k_in, B, len(slots), c_s, kf, self, dt_s, inv)
    f[60] = gl[4]
    f[62] = gl[6]
    return bf16(f)


def q_of(logits, nvalid, slot, eps, B):
    """q(target) of the mixture from one row of FP32 logits (slot -1: not a candidate)."""
    L = np.asarray(logits, np.float32)
    mx = L[ESCAPE]
    for j in range(nvalid):
        mx = max(mx, L[j])
    ex = [np.exp(np.float64(np.float32(L[j] - mx))) for j in range(nvalid)]
    esc = np.exp(np.float64(np.float32(L[ESCAPE] - mx)))
    S = esc
    for x in ex:
        S += x
    w = 1.0 - np.float64(np.float32(eps))
    q = (w * (esc / S) + np.float64(np.float32(eps))) / B
    if slot >= 0:
        q += w * ex[slot] / S
    return q


def draw(logits, nvalid, slots, x0, x1, eps, B):
    """Block drawn with record words (x0 = choice, x1 = uniform block)."""
    L = np.asarray(logits, np.float32)
    mx = L[ESCAPE]
    for j in range(nvalid):
        mx = max(mx, L[j])
    S = np.exp(np.float64(np.float32(L[ESCAPE] - mx)))
    for j in range(nvalid):
        S += np.exp(np.float64(np.float32(L[j] - mx)))
    w = 1.0 - np.float64(np.float32(eps))
    u = np.float64(x0) * 2.0 ** -32
    acc = 0.0
    for j in range(nvalid):
        acc += w * np.exp(np.float64(np.float32(L[j] - mx))) / S
        if u < acc:
            return slots[j][0]
    return int((int(x1) * B) >> 32)
