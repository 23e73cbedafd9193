"""CPU oracle of the learned preconditioner (numpy/scipy, FP64).

TEST INFRASTRUCTURE ONLY.  tests/ use it as the checker of the GPU network
(ofeli_b200/csrc/learned.cu); the product never imports it.  The learned
preconditioner has no counterpart in OFELI, so this restates the network as
the library defines it (the comment block at the top of learned.cu):

    d_i   = sqrt|a_ii|,  a~_ij = a_ij / (d_i d_j) (i != j), 0 on the diagonal
    f_i   = (1, deg_i/16, sum_j |a~_ij|, log a_ii - mean_k log a_kk)
    h0    = relu(f W_in + b_in)
    layer h_{l+1} = relu([h_l | A~ h_l] W_l + b_l) + h_l          (4 layers)
    head  G_ii = softplus(v.h_i + c) / d_i
          G_ij = a~_ij (u . (h_i o h_j)) / d_j        (j < i, a~_ij != 0)
    M     = G^T G
    loss  kind 0: mean_p ||M r_p - e_p||^2 / ||e_p||^2
          kind 1: log(T/n) - (2/n) sum_i log G_ii,
                  T = (1/P) sum_p (G e_p . G r_p) n / ||e_p||^2   (Kaporin number)

and its gradient by reverse-mode differentiation written out by hand.
With bf16=True the values the GPU keeps in BF16 (pre-activations z, hidden
states h, the layer input [h | A~ h], the layer weights and the BF16 copy of
dZ fed to the data-gradient product) are rounded to BF16 at the same points,
so that the oracle and the GPU differ only by FP32 vs FP64 accumulation.
With bf16=False the oracle is plain FP64 and is checked against finite
differences.
"""
import numpy as np
import scipy.sparse as sp

HID, NFEAT, NLAYER = 64, 4, 4
P_WIN = 0
P_BIN = P_WIN + NFEAT * HID
P_W = P_BIN + HID
P_B = P_W + NLAYER * 2 * HID * HID
P_U = P_B + NLAYER * HID
P_V = P_U + HID
P_C = P_V + HID
NPARAM = P_C + 1


def round_bf16(x):
    """Round-to-nearest-even of float values to BF16 (returned as float64)."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(P):
    P = np.asarray(P, dtype=np.float64)
    return {
        "W_in": P[P_WIN:P_BIN].reshape(NFEAT, HID),
        "b_in": P[P_BIN:P_W],
        "W": [P[P_W + l * 2 * HID * HID:P_W + (l + 1) * 2 * HID * HID].reshape(2 * HID, HID)
              for l in range(NLAYER)],
        "b": [P[P_B + l * HID:P_B + (l + 1) * HID] for l in range(NLAYER)],
        "u": P[P_U:P_V], "v": P[P_V:P_C], "c": P[P_C],
    }


class Graph:
    """Scaled graph and node features of a CSR matrix (0-based columns)."""

    def __init__(self, row_ptr, col, val):
        self.rp = np.asarray(row_ptr, dtype=np.int64)
        self.col = np.asarray(col, dtype=np.int64)
        self.val = np.asarray(val, dtype=np.float64)
        n = self.n = len(self.rp) - 1
        self.rows = np.repeat(np.arange(n), np.diff(self.rp))
        diag = self.col == self.rows
        dval = np.zeros(n)
        dval[self.rows[diag]] = self.val[diag]
        self.dsq = np.sqrt(np.abs(dval)).astype(np.float32).astype(np.float64)
        at = np.where(diag, 0.0, self.val / (self.dsq[self.rows] * self.dsq[self.col]))
        self.at = at.astype(np.float32).astype(np.float64)
        self.Atil = sp.csr_matrix((self.at, self.col, self.rp), shape=(n, n))
        deg = np.bincount(self.rows[~diag], minlength=n)
        rs = np.bincount(self.rows, weights=np.abs(self.at), minlength=n)
        logd = 2.0 * np.log(self.dsq)
        self.feat = np.stack([np.ones(n), deg / 16.0, rs, logd - logd.mean()], axis=1)
        self.lower = (self.col < self.rows) & (self.at != 0.0)   # off-diagonal factor entries
        self.diag = diag


def forward(g, P, bf16=True):
    """Activations and the factor G (values at the CSR positions)."""
    rb = round_bf16 if bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    p = split_params(P)
    s0 = g.feat @ p["W_in"] + p["b_in"]
    z = [rb(s0)]
    h = [rb(np.maximum(s0, 0.0))]
    cat = []
    for l in range(NLAYER):
        c = np.concatenate([h[l], rb(g.Atil @ h[l])], axis=1)
        cat.append(c)
        s = c @ rb(p["W"][l]) + p["b"][l]
        z.append(rb(s))
        h.append(rb(np.maximum(s, 0.0) + h[l]))
    H = h[NLAYER]
    sdiag = H @ p["v"] + p["c"]
    gv = np.zeros(len(g.col))
    d = g.diag
    gv[d] = np.maximum(np.logaddexp(0.0, sdiag[g.rows[d]]), 1e-20) / g.dsq[g.rows[d]]
    lo = g.lower
    score = (H[g.rows[lo]] * H[g.col[lo]]) @ p["u"]
    gv[lo] = g.at[lo] * score / g.dsq[g.col[lo]]
    return {"z": z, "h": h, "cat": cat, "sdiag": sdiag, "score": score, "g": gv, "p": p}


def factor_matrix(g, gv):
    keep = g.diag | g.lower
    return sp.csr_matrix((np.where(keep, gv, 0.0), g.col, g.rp), shape=(g.n, g.n))


def apply(g, gv, R):
    """M R = G^T (G R); R is n x P (columns are pairs)."""
    G = factor_matrix(g, gv)
    return G.T @ (G @ R)


def loss_and_grad(g, P, R, E, bf16=True, kind=1):
    """Loss over the pairs (R, E given pair-major, P x n) and its gradient."""
    rb = round_bf16 if bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    f = forward(g, P, bf16)
    p = f["p"]
    R = np.asarray(R, dtype=np.float64).T
    E = np.asarray(E, dtype=np.float64).T
    npairs = R.shape[1]
    n = g.n
    G = factor_matrix(g, f["g"])
    Z = G @ R
    en = (E * E).sum(axis=0)
    en[en == 0] = 1.0
    if kind == 0:
        Y = G.T @ Z
        w = 1.0 / (en * npairs)
        loss = float((((Y - E) ** 2) * w).sum())
        dY = 2.0 * (Y - E) * w
    else:
        GE = G @ E
        T = float(((Z * GE).sum(axis=0) * n / (en * npairs)).sum())
        loss = np.log(T / n) - 2.0 * np.log(f["g"][g.diag]).sum() / n
        dY = E * (n / (en * npairs * T))
    dZ = G @ dY
    rows, col = g.rows, g.col
    dG = np.zeros(len(col))
    keep = g.diag | g.lower
    dG[keep] = ((dY[col[keep]] * Z[rows[keep]]).sum(1) + (dZ[rows[keep]] * R[col[keep]]).sum(1))
    if kind != 0:
        dG[g.diag] -= 2.0 / (n * f["g"][g.diag])
    H = f["h"][NLAYER]
    grad = np.zeros(NPARAM)
    # head
    d = g.diag
    di = rows[d]
    sig = 1.0 / (1.0 + np.exp(-f["sdiag"][di]))
    dsd = dG[d] * sig / g.dsq[di]
    lo = g.lower
    dS = dG[lo] * g.at[lo] / g.dsq[col[lo]]
    li, lj = rows[lo], col[lo]
    grad[P_U:P_V] = (dS[:, None] * H[li] * H[lj]).sum(0)
    grad[P_V:P_C] = (dsd[:, None] * H[di]).sum(0)
    grad[P_C] = dsd.sum()
    dH = np.zeros_like(H)
    np.add.at(dH, di, dsd[:, None] * p["v"][None, :])
    np.add.at(dH, li, dS[:, None] * p["u"][None, :] * H[lj])
    np.add.at(dH, lj, dS[:, None] * p["u"][None, :] * H[li])
    # layers
    for l in range(NLAYER - 1, -1, -1):
        dz = dH * (f["z"][l + 1] > 0)
        c = f["cat"][l]
        # the weight and bias gradients, like the data product, take dz in
        # BF16 (the GPU's tensor-core operand)
        grad[P_W + l * 2 * HID * HID:P_W + (l + 1) * 2 * HID * HID] = (c.T @ rb(dz)).ravel()
        grad[P_B + l * HID:P_B + (l + 1) * HID] = rb(dz).sum(0)
        dcat = rb(dz) @ rb(p["W"][l]).T
        dH = dH + dcat[:, :HID] + g.Atil @ dcat[:, HID:]
    dz0 = dH * (f["z"][0] > 0)
    grad[P_WIN:P_BIN] = (g.feat.T @ dz0).ravel()
    grad[P_BIN:P_W] = dz0.sum(0)
    return loss, grad


def init_params(seed):
    """The library's initial parameters (lp_init_params): Xavier-uniform
    weights from a splitmix-style counter hash, zero biases, u = v = 0 and
    softplus(c) = 1, so that M starts as Jacobi."""
    t = np.arange(NPARAM, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)) + (t + np.uint64(1)) * np.uint64(
            0xD1B54A32D192ED03)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u01 = ((z >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)
    P = np.zeros(NPARAM, dtype=np.float32)
    idx = np.arange(NPARAM)
    a = np.sqrt(np.float32(6.0) / np.float32(NFEAT + HID))
    P[idx < P_BIN] = ((2 * u01 - 1) * a)[idx < P_BIN]
    wm = (idx >= P_W) & (idx < P_B)
    P[wm] = ((2 * u01 - 1) * np.sqrt(np.float32(6.0) / np.float32(3 * HID)) * np.float32(0.5))[wm]
    P[P_C] = np.float32(0.54132485)
    return P
