"""CPU restatement of the learned scheme switch -- test infrastructure only
(the checker of the GPU kernels in ocfd_learned.cu; never called by the
library).

* features(): the 14 switch features of interior cells of a periodic state,
  from the plain sensor's 7-point stencil (Comput_P and
  Comput_Scheme_point_Jameson, src/OCFD_Schemes_hybrid_auto.cu:48-68,
  611-703: P = p00 d T, the sensor term |P- - 2P0 + P+| / (P- + 2P0 + P+)
  per direction), plus first differences and the same terms of density.
* forward_backward(): the network 14 -> 32 -> 32 -> 1 (ReLU) in FP64, the
  summed binary cross-entropy with logits (positives weighted pos_w) and its
  gradient with respect to the network parameters, by hand-written
  back-propagation.
* logits_bf16(): the forward pass as the tensor-core kernel forms it: inputs,
  weights and first-layer activations rounded to BF16 (nearest even), FP32
  accumulation, output layer in FP32.
"""
import numpy as np

NIN, NH = 14, 32
OFF_MU, OFF_SG, OFF_W1 = 0, 14, 28
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OFF_MU:OFF_MU + NIN], w[OFF_SG:OFF_SG + NIN], w[OFF_W1:OFF_B1].reshape(NH, NIN),
            w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH), w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def features(d, T, p00):
    """Features of every interior cell of a periodic field (arrays [z][y][x]),
    in x-fastest order; also the plain sensor value dp of each cell."""
    d = np.asarray(d, np.float64)
    P = p00 * d * np.asarray(T, np.float64)
    cols, dp = [], None
    s2p, s1p, s2d, s1d = [], [], [], []
    for ax in (2, 1, 0):                       # x, y, z
        Pm, Pp = np.roll(P, 1, axis=ax), np.roll(P, -1, axis=ax)
        den = Pm + 2 * P + Pp
        t = np.abs(-Pm + 2 * P - Pp) / den
        dp = t if dp is None else dp + t
        s2p.append(t); s1p.append((Pp - Pm) / den)
        Dm, Dp = np.roll(d, 1, axis=ax), np.roll(d, -1, axis=ax)
        dd = Dm + 2 * d + Dp
        s2d.append(np.abs(-Dm + 2 * d - Dp) / dd); s1d.append((Dp - Dm) / dd)
    f = [x.astype(np.float32) for x in s2p + s1p + s2d + s1d]
    f.append(f[0] + f[1] + f[2])
    f.append(f[6] + f[7] + f[8])
    return np.stack([x.ravel() for x in f], axis=1), dp.ravel()


def _relu(x):
    return np.maximum(x, 0.0)


def forward_backward(w, feat, label, pos_w=1.0):
    """(summed loss, gradient of the network part of w (from W1 on))."""
    mu, sg, W1, b1, W2, b2, W3, b3 = unpack(w)
    x = (np.asarray(feat, np.float64) - mu) / sg
    y = np.asarray(label, np.float64)
    z1 = x @ W1.T + b1
    h1 = _relu(z1)
    z2 = h1 @ W2.T + b2
    h2 = _relu(z2)
    z3 = h2 @ W3 + b3
    wt = np.where(y > 0.5, pos_w, 1.0)
    loss = np.sum(wt * (np.maximum(z3, 0) - z3 * y + np.log1p(np.exp(-np.abs(z3)))))
    d3 = wt * (1.0 / (1.0 + np.exp(-z3)) - y)
    d2 = (d3[:, None] * W3[None, :]) * (z2 > 0)
    d1 = (d2 @ W2) * (z1 > 0)
    g = np.concatenate([(d1.T @ x).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0),
                        (d3[:, None] * h2).sum(0), [d3.sum()]])
    return loss, g


def bf16(a):
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def logits_bf16(w, feat):
    mu, sg, W1, b1, W2, b2, W3, b3 = [np.asarray(v, np.float32) for v in unpack(w)]
    x = bf16((np.asarray(feat, np.float32) - mu) / sg)
    z1 = x.astype(np.float64) @ bf16(W1).T.astype(np.float64) + b1
    h1 = bf16(np.maximum(z1, 0).astype(np.float32))
    z2 = h1.astype(np.float64) @ bf16(W2).T.astype(np.float64) + b2
    h2 = np.maximum(z2, 0)
    return (h2 @ W3.astype(np.float64) + b3).astype(np.float32)
