"""CPU restatement of the learned step-size proposer's network (test
infrastructure only: the parity checker of the GPU training and inference
kernels; never part of the product path).

The reference has no learned proposer (its controller restarts every
measurement interval at measure_every / n_subdivisions, PiFlux.cpp:104-110),
so there is nothing upstream to pin against.  This oracle is pinned
mathematically instead: with ``emulate=False`` it is the exact float64
gradient of the float64 network, checked against central finite differences
in the CPU tests; with ``emulate=True`` it applies the BF16 roundings the GPU
applies (inputs, weights, hidden activations, back-propagated pre-activation
gradients) so the GPU's gradients and predictions can be compared with it.

Network: 8 -> 64 -> 64 -> 64 -> 1, SiLU after the first three layers.
Parameter layout (flat float32, the C ABI's hhg_mlp.params): w1[64][8], b1,
w2[64][64], b2, w3[64][64], b3, w4[64], b4.  Records: HIST_FIELDS floats, the
8 raw inputs then the target level T.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 8, 64
LAYOUT = [("w1", (64, 8)), ("b1", (64,)), ("w2", (64, 64)), ("b2", (64,)),
          ("w3", (64, 64)), ("b3", (64,)), ("w4", (64,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in LAYOUT)


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest, ties to even) and
    return them as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).reshape(a.shape)


def unpack(flat) -> dict:
    flat = np.asarray(flat)
    out, o = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def pack(t: dict) -> np.ndarray:
    return np.concatenate([np.asarray(t[name], dtype=np.float64).reshape(-1)
                           for name, _ in LAYOUT])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _inputs(records, in_mu, in_isig, emulate):
    r = np.asarray(records)
    if emulate:
        x = (r[:, :N_IN].astype(np.float32) - np.float32(in_mu)) * np.float32(in_isig)
        return bf16(x).astype(np.float64)
    return (r[:, :N_IN].astype(np.float64) - np.asarray(in_mu, np.float64)) * \
        np.asarray(in_isig, np.float64)


def _targets(records, out_mu, out_sigma, emulate):
    r = np.asarray(records)
    if emulate:
        isig = np.float32(1.0) / np.float32(out_sigma)
        return ((r[:, N_IN].astype(np.float32) - np.float32(out_mu)) * isig).astype(np.float64)
    return (r[:, N_IN].astype(np.float64) - out_mu) / out_sigma


def silu_bf16_tanh(z):
    """The inference kernel's activation: z rounded to BF16, h = z / 2,
    y = h + h tanh(h) with tanh and the fused multiply-add rounded to BF16
    (the hardware tanh is an approximation within a few BF16 units of the
    rounded exact value, so this emulation is close but not bit-exact)."""
    h = bf16(bf16(np.asarray(z, np.float32)) * np.float32(0.5))
    t = bf16(np.tanh(h.astype(np.float64)).astype(np.float32))
    return bf16((h.astype(np.float64) + h.astype(np.float64) * t).astype(np.float32))


def forward(flat, records, in_mu, in_isig, emulate=True, act="fp32") -> dict:
    """Intermediates and the standardised output y (float64 arithmetic).
    act = "fp32": SiLU in FP32 then BF16 rounding (training forward);
    act = "bf16_tanh": the inference kernel's BF16 tanh form."""
    p = unpack(np.asarray(flat, np.float32) if emulate else np.asarray(flat, np.float64))
    rnd = (lambda a: bf16(a).astype(np.float64)) if emulate else (lambda a: np.asarray(a, np.float64))
    W = {k: rnd(p[k]) for k in ("w1", "w2", "w3", "w4")}
    b = {k: np.asarray(p[k], np.float64) for k in ("b1", "b2", "b3", "b4")}
    x = _inputs(records, in_mu, in_isig, emulate)
    if emulate and act == "bf16_tanh":
        def sact(z):
            return silu_bf16_tanh(z).astype(np.float64)
    else:
        def sact(z):
            return rnd(silu(z))
    z1 = x @ W["w1"].T + b["b1"]
    h1 = sact(z1)
    z2 = h1 @ W["w2"].T + b["b2"]
    h2 = sact(z2)
    z3 = h2 @ W["w3"].T + b["b3"]
    h3 = sact(z3)
    y = h3 @ W["w4"] + b["b4"][0]
    return dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3, y=y, W=W)


def predict(flat, records, in_mu, in_isig, out_mu, out_sigma, emulate=True,
            act="fp32") -> np.ndarray:
    """Predicted level T (de-standardised)."""
    return forward(flat, records, in_mu, in_isig, emulate, act)["y"] * out_sigma + out_mu


def loss_and_grad(flat, records, in_mu, in_isig, out_mu, out_sigma, emulate=True):
    """Mean squared error of the standardised level and its gradient with
    respect to the flat parameters (the GPU's hhg_mlp_gradients)."""
    f = forward(flat, records, in_mu, in_isig, emulate)
    rnd = (lambda a: bf16(a).astype(np.float64)) if emulate else (lambda a: a)
    t = _targets(records, out_mu, out_sigma, emulate)
    n = t.shape[0]
    d = f["y"] - t
    loss = float(np.mean(d * d))
    gy = 2.0 * d / n
    W = f["W"]
    g = {}
    g["w4"] = f["h3"].T @ gy
    g["b4"] = np.array([gy.sum()])
    dz3 = rnd(gy[:, None] * W["w4"][None, :] * dsilu(f["z3"]))
    g["w3"] = dz3.T @ f["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = rnd((dz3 @ W["w3"]) * dsilu(f["z2"]))
    g["w2"] = dz2.T @ f["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = rnd((dz2 @ W["w2"]) * dsilu(f["z1"]))
    g["w1"] = dz1.T @ f["x"]
    g["b1"] = dz1.sum(0)
    return loss, pack(g)
