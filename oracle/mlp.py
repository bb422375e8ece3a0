"""CPU oracle (test infrastructure) of the share network: numpy forward and backward.

Layout of the flat FP32 parameter vector (as in libits): W1[128x64] b1[128] W2[128x128]
b2[128] W3[128x128] b3[128] w4[128] b4[1], W[o][i] = weight from input i to output o.

``forward``/``gradient`` with ``bf16=True`` round to bfloat16 at the same points as the
GPU kernels (features, weights, hidden activations, output weights, the dZ operands of the
backward products) and accumulate in float64; with ``bf16=False`` everything is float64,
which is what the finite-difference check in the CPU tests differentiates.
"""
import numpy as np

N_IN, N_HID = 64, 128
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("w4", (N_HID,)), ("b4", (1,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], np.float64).reshape(shape)
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


K0, K1 = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks & Gimpel 2016): z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * z * z)


def init_params(seed=0):
    """He-style initialisation (uniform, fan-in scaled), zero biases."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("b"):
            d[name] = np.zeros(shape)
        else:
            fan_in = shape[-1] if len(shape) == 2 else N_HID
            d[name] = rng.uniform(-1, 1, shape) * np.sqrt(3.0 / fan_in)
    return pack(d).astype(np.float32)


def _forward(P, X, rnd):
    r = bf16 if rnd else (lambda a: np.asarray(a, np.float64))
    W = {k: (r(v) if k[0] == "W" or k == "w4" else v) for k, v in unpack(P).items()}
    x = r(X)
    z1 = x @ W["W1"].T + W["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W["W2"].T + W["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ W["W3"].T + W["b3"]
    h3 = r(gelu(z3))
    out = h3 @ W["w4"] + W["b4"][0]
    return out, (W, x, z1, h1, z2, h2, z3, h3)


def forward(P, X, bf16_round=True):
    return _forward(P, X, bf16_round)[0]


def gradient(P, X, y, bf16_round=True):
    """Gradient of mean((out - y)^2) with respect to the flat parameters, and the loss."""
    r = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    out, (W, x, z1, h1, z2, h2, z3, h3) = _forward(P, X, bf16_round)
    n = X.shape[0]
    e = out - y
    d = 2.0 * e / n
    g = {}
    g["w4"] = h3.T @ d
    g["b4"] = np.array([d.sum()])
    dz3 = r(d[:, None] * W["w4"][None, :] * gelu_grad(z3))
    g["W3"] = dz3.T @ h2
    g["b3"] = dz3.sum(0)
    dz2 = r((dz3 @ W["W3"]) * gelu_grad(z2))
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = r((dz2 @ W["W2"]) * gelu_grad(z1))
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return pack(g), float(np.mean(e * e))


def adam(P, M, V, G, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    M = b1 * M + (1 - b1) * G
    V = b2 * V + (1 - b2) * G * G
    P = P - lr * (M / (1 - b1 ** step)) / (np.sqrt(V / (1 - b2 ** step)) + eps)
    return P, M, V
