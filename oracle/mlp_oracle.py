"""ORACLE — test infrastructure only: an FP64 numpy restatement of the learned
w-kernel network, its input features and its gradients, used to check the
project's CUDA training and inference kernels (csrc/k_mlp.cu).

Network (no counterpart in the reference): 21 input features -> 128 -> 128 ->
128 (SiLU) -> 2 (a complex tap, scaled by out_scale).  Features of a tap
(w, du, dv, tx, ty) for support K, with p = tx - K/2 - du and q = ty - K/2 - dv
(the tap's offset from the visibility, in cells):
    w / wmax, 2 du - 1, 2 dv - 1, p / (K/2), q / (K/2),
    cos(pi k p / (K/2 + 1)), sin(pi k p / (K/2 + 1))  for k = 1..4,
    cos(pi k q / (K/2 + 1)), sin(pi k q / (K/2 + 1))  for k = 1..4,
padded with zeros to 32.  Parameter layout (float32 on the device):
    W1[32][128], b1[128], W2[128][128], b2[128], W3[128][128], b3[128],
    W4[128][2], b4[2].
"""
import numpy as np

H, FIN, NFEAT = 128, 32, 21
SIZES = [("W1", (FIN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
         ("b3", (H,)), ("W4", (H, 2)), ("b4", (2,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(flat):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(params):
    return np.concatenate([np.asarray(params[name], np.float64).ravel() for name, _ in SIZES])


def features(w, du, dv, tx, ty, ksize, wmax):
    w, du, dv, tx, ty = (np.asarray(a, np.float64) for a in (w, du, dv, tx, ty))
    half = ksize / 2.0
    p = tx - half - du
    q = ty - half - dv
    f = np.zeros(w.shape + (FIN,))
    f[..., 0] = w / wmax
    f[..., 1] = 2 * du - 1
    f[..., 2] = 2 * dv - 1
    f[..., 3] = p / half
    f[..., 4] = q / half
    for k in range(1, 5):
        f[..., 5 + 2 * (k - 1)] = np.cos(np.pi * k * p / (half + 1))
        f[..., 6 + 2 * (k - 1)] = np.sin(np.pi * k * p / (half + 1))
        f[..., 13 + 2 * (k - 1)] = np.cos(np.pi * k * q / (half + 1))
        f[..., 14 + 2 * (k - 1)] = np.sin(np.pi * k * q / (half + 1))
    return f


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, f):
    P = params
    z1 = f @ P["W1"] + P["b1"]
    h1 = silu(z1)
    z2 = h1 @ P["W2"] + P["b2"]
    h2 = silu(z2)
    z3 = h2 @ P["W3"] + P["b3"]
    h3 = silu(z3)
    y = h3 @ P["W4"] + P["b4"]
    return y, (f, z1, h1, z2, h2, z3, h3)


def loss_and_grads(params, f, target):
    """L = (1/B) sum |y - target|^2 over both components; analytic gradients."""
    P = params
    y, (f, z1, h1, z2, h2, z3, h3) = forward(P, f)
    B = f.shape[0]
    d = y - target
    loss = float(np.sum(d * d) / B)
    dy = 2.0 * d / B
    g = {"W4": h3.T @ dy, "b4": dy.sum(0)}
    dz3 = (dy @ P["W4"].T) * dsilu(z3)
    g["W3"], g["b3"] = h2.T @ dz3, dz3.sum(0)
    dz2 = (dz3 @ P["W3"].T) * dsilu(z2)
    g["W2"], g["b2"] = h1.T @ dz2, dz2.sum(0)
    dz1 = (dz2 @ P["W2"].T) * dsilu(z1)
    g["W1"], g["b1"] = f.T @ dz1, dz1.sum(0)
    return loss, g


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    P = {}
    for name, shape in SIZES:
        if name.startswith("W"):
            fan_in = NFEAT if name == "W1" else shape[0]
            P[name] = rng.normal(0, np.sqrt(2.0 / fan_in), size=shape)
            if name == "W1":
                P[name][NFEAT:] = 0.0
        else:
            P[name] = np.zeros(shape)
    return P
