"""CPU restatement (float64) of the learned projection of the proposal matcher.

TEST INFRASTRUCTURE ONLY: the checker for the GPU forward, loss and gradient kernels of
eth-v3d-lgpl_b200/csrc/v3dm_proposal.cu.  The projection has no counterpart in the reference,
so this file restates its definition:
  x = u / 512,  h = relu(W1b x + b1),  z = W2b h + b2,  zn = z / |z|,
  s_kl = zn(a_k) . zn(p_l) / T,
  L = 1/(2B) sum_k (lse_l s_kl - s_kk) + 1/(2B) sum_l (lse_k s_kl - s_ll),
where W1b, W2b are the BF16 roundings (nearest even) of the FP32 master weights, and returns
L and dL/d(parameters) in the flat layout W1[64][128], b1[64], W2[32][64], b2[32]."""
import numpy as np

N_IN, N_HID, N_OUT = 128, 64, 32
OFF_B1 = N_HID * N_IN
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_OUT * N_HID
N_PARAMS = OFF_B2 + N_OUT


def bf16_round(w: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 value (ties to even), returned as float32."""
    b = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray, bf16: bool = True):
    """Layers of a parameter vector; bf16=False keeps the weights unrounded (float64), for
    finite-difference checks of the formulas."""
    if bf16:
        p = np.asarray(params, np.float32)
        W1 = bf16_round(p[:OFF_B1]).astype(np.float64)
        W2 = bf16_round(p[OFF_W2:OFF_B2]).astype(np.float64)
    else:
        p = np.asarray(params, np.float64)
        W1, W2 = p[:OFF_B1], p[OFF_W2:OFF_B2]
    return (W1.reshape(N_HID, N_IN), p[OFF_B1:OFF_W2].astype(np.float64), W2.reshape(N_OUT, N_HID),
            p[OFF_B2:].astype(np.float64))


def forward(params: np.ndarray, desc: np.ndarray, bf16: bool = True):
    W1, b1, W2, b2 = unpack(params, bf16)
    x = np.asarray(desc, np.float64) / 512.0
    pre = x @ W1.T + b1
    h = np.maximum(pre, 0.0)
    z = h @ W2.T + b2
    nrm = np.sqrt((z * z).sum(1))
    zn = z / np.maximum(nrm, 1e-12)[:, None]
    return x, h, z, nrm, zn


def embed(params: np.ndarray, desc: np.ndarray) -> np.ndarray:
    return forward(params, desc)[4]


def loss_grad(params: np.ndarray, anchors: np.ndarray, positives: np.ndarray, T: float, bf16: bool = True):
    W1, b1, W2, b2 = unpack(params, bf16)
    B = anchors.shape[0]
    x, h, z, nrm, zn = forward(params, np.concatenate([anchors, positives]), bf16)
    za, zp = zn[:B], zn[B:]
    S = za @ zp.T / T
    lse_r = np.log(np.exp(S - S.max(1, keepdims=True)).sum(1)) + S.max(1)
    lse_c = np.log(np.exp(S - S.max(0, keepdims=True)).sum(0)) + S.max(0)
    d = np.diag(S)
    loss = ((lse_r - d).sum() + (lse_c - d).sum()) / (2 * B)
    G = (np.exp(S - lse_r[:, None]) + np.exp(S - lse_c[None, :]) - 2 * np.eye(B)) / (2 * B)
    dza = G @ zp / T
    dzp = G.T @ za / T
    dzn = np.concatenate([dza, dzp])
    dz = (dzn - zn * (zn * dzn).sum(1, keepdims=True)) / np.maximum(nrm, 1e-12)[:, None]
    dh = (dz @ W2) * (h > 0)
    grad = np.concatenate([(dh.T @ x).reshape(-1), dh.sum(0), (dz.T @ h).reshape(-1), dz.sum(0)])
    return float(loss), grad


def loss_only(params, anchors, positives, T, bf16: bool = True):
    """The loss without the gradient (for finite-difference checks of loss_grad)."""
    B = anchors.shape[0]
    zn = forward(params, np.concatenate([anchors, positives]), bf16)[4]
    S = zn[:B] @ zn[B:].T / T
    lse_r = np.log(np.exp(S - S.max(1, keepdims=True)).sum(1)) + S.max(1)
    lse_c = np.log(np.exp(S - S.max(0, keepdims=True)).sum(0)) + S.max(0)
    d = np.diag(S)
    return float(((lse_r - d).sum() + (lse_c - d).sum()) / (2 * B))


def init_params(seed: int) -> np.ndarray:
    """A float32 parameter vector for tests (He-uniform weights, small random biases)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[:OFF_B1] = rng.uniform(-np.sqrt(6 / N_IN), np.sqrt(6 / N_IN), OFF_B1)
    p[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, N_HID)
    p[OFF_W2:OFF_B2] = rng.uniform(-np.sqrt(6 / N_HID), np.sqrt(6 / N_HID), N_OUT * N_HID)
    p[OFF_B2:] = rng.uniform(-0.1, 0.1, N_OUT)
    return p
