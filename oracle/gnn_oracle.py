"""CPU restatement (float64 numpy) of the graph-network preconditioner of the
learned form: near-field pattern, features, forward pass, objective and the
hand-written backward pass, for checking the CUDA kernels.

Test infrastructure only: imported by tests/ and nothing else.  There is no
reference counterpart (the reference solves its VIE systems by dense LU only,
libhmat HMatrix::LUFactorize / LUSolve); the backward pass here is pinned
against central finite differences of the forward pass in the CPU tests.

Network: h0 = relu(W0 f + b0); three layers of
  z_e = Wmh h_j + Wme g_e + bm, agg_i = mean_{e in row i} relu(z_e),
  h_i <- h_i + relu(Wuh h_i + Wua agg_i + bu);
edge readout y_e = relu(Wri h_i + Wrj h_j + Wrg g_e + br), o_e = Wo y_e + bo,
  c = CMAX (tanh o0 + i tanh o1), s = smax (tanh o2 + i tanh o3 / 2),
  m_ij = [delta_ij + c - [i != j] s A_ij / A_ii] / A_jj,
with smax = SREL / max(SREL, rho(K1)), rho(K1) a 16-step power-iteration
estimate (four seeded start vectors, as on the device) of the spectral radius
of K1 (K1_ij = A_ij / A_jj off the diagonal on the pattern).

Parameter layout (floats, in order): W0 (64x8), b0 (64), per layer l<3:
Wmh (64x64), Wme (64x8), bm (64), Wuh (64x64), Wua (64x64), bu (64); then
Wri (64x64), Wrj (64x64), Wrg (64x8), br (64), Wo (4x64), bo (4).  Matrices
are row-major (out x in).
"""
import numpy as np

GW, GF, GE, GL, GO = 64, 8, 8, 3, 4
CMAX, SREL, POWER_ITERS = 0.1, 0.7, 16


def layout():
    off = {}
    o = 0

    def take(name, n):
        nonlocal o
        off[name] = (o, n)
        o += n

    take("W0", GW * GF)
    take("b0", GW)
    for l in range(GL):
        take(f"Wmh{l}", GW * GW)
        take(f"Wme{l}", GW * GE)
        take(f"bm{l}", GW)
        take(f"Wuh{l}", GW * GW)
        take(f"Wua{l}", GW * GW)
        take(f"bu{l}", GW)
    take("Wri", GW * GW)
    take("Wrj", GW * GW)
    take("Wrg", GW * GE)
    take("br", GW)
    take("Wo", GO * GW)
    take("bo", GO)
    return off, o


SHAPES = {"W0": (GW, GF), "b0": (GW,), "Wri": (GW, GW), "Wrj": (GW, GW), "Wrg": (GW, GE), "br": (GW,),
          "Wo": (GO, GW), "bo": (GO,)}
for _l in range(GL):
    SHAPES.update({f"Wmh{_l}": (GW, GW), f"Wme{_l}": (GW, GE), f"bm{_l}": (GW,), f"Wuh{_l}": (GW, GW),
                   f"Wua{_l}": (GW, GW), f"bu{_l}": (GW,)})


def unpack(flat):
    off, _ = layout()
    return {k: np.asarray(flat[o:o + n], dtype=np.float64).reshape(SHAPES[k]) for k, (o, n) in off.items()}


def pack(d):
    off, total = layout()
    out = np.zeros(total)
    for k, (o, n) in off.items():
        out[o:o + n] = np.asarray(d[k]).reshape(-1)
    return out


def bf_vertices(faces):
    """5 vertex indices (QP, V1, V2, V3, QM) of each basis function from the
    9-column face table (iV1, iV2, iV3, iQP, iQM, iPTet, iMTet, PIndex, MIndex)."""
    f = np.asarray(faces)
    return np.stack([f[:, 3], f[:, 0], f[:, 1], f[:, 2], f[:, 4]], axis=1)


def pattern(faces):
    """CSR (rowptr, col) of basis-function pairs with at least one common
    vertex, self pairs included, columns sorted; and the reverse-edge map."""
    bv = bf_vertices(faces)
    N = len(bv)
    inc = {}
    for a in range(N):
        for v in set(bv[a].tolist()):
            inc.setdefault(v, []).append(a)
    rows = [set([i]) for i in range(N)]
    for lst in inc.values():
        for a in lst:
            rows[a].update(lst)
    rowptr = np.zeros(N + 1, np.int64)
    cols = []
    for i in range(N):
        r = sorted(rows[i])
        cols.extend(r)
        rowptr[i + 1] = rowptr[i] + len(r)
    col = np.array(cols, np.int64)
    pos = {(i, int(col[e])): e for i in range(N) for e in range(rowptr[i], rowptr[i + 1])}
    etr = np.array([pos[(int(col[e]), i)] for i in range(N) for e in range(rowptr[i], rowptr[i + 1])], np.int64)
    return rowptr, col, etr


def features(V, faces, A, omega, rowptr, col):
    """Node (N x 8) and edge (E x 8) features, the ratios A_ij / A_ii per edge
    and 1/A_jj, as the device feature kernel computes them."""
    f = np.asarray(faces)
    N = len(f)
    bv = bf_vertices(f)
    P1, P2, P3 = V[f[:, 0]], V[f[:, 1]], V[f[:, 2]]
    cen = (P1 + P2 + P3) / 3.0
    area = 0.5 * np.linalg.norm(np.cross(P2 - P1, P3 - P1), axis=1)
    radius = np.max(np.stack([np.linalg.norm(cen - V[f[:, k]], axis=1) for k in (3, 0, 1, 2, 4)]), axis=0)
    h = radius.mean()
    d = np.diag(A)
    am = np.abs(d)
    deg = np.diff(rowptr)
    F = np.zeros((N, GF))
    F[:, 0] = 1.0
    F[:, 1] = d.real / am
    F[:, 2] = d.imag / am
    F[:, 3] = omega * h
    F[:, 4] = area / h ** 2
    F[:, 5] = radius / h
    F[:, 6] = deg / 100.0
    F[:, 7] = np.log10(am) * 0.1
    rows = np.repeat(np.arange(N), deg)
    r = A[rows, col] / d[rows]
    rt = A[col, rows] / d[col]
    ncv = np.array([np.sum(bv[i][:, None] == bv[j][None, :]) for i, j in zip(rows, col)])
    dist = np.linalg.norm(cen[rows] - cen[col], axis=1)
    Ef = np.zeros((len(col), GE))
    Ef[:, 0] = r.real
    Ef[:, 1] = r.imag
    Ef[:, 2] = rt.real
    Ef[:, 3] = rt.imag
    Ef[:, 4] = dist / h
    Ef[:, 5] = ncv / 5.0
    Ef[:, 6] = (rows == col).astype(float)
    Ef[:, 7] = np.abs(r)
    return F, Ef, r, 1.0 / d


def relu(x):
    return np.maximum(x, 0.0)


def seeded_vectors(N, nv=4):
    """The device's start vectors: 64-bit LCG, uniform in [-0.5, 0.5), re/im interleaved."""
    s = 0x9E3779B97F4A7C15
    M64 = (1 << 64) - 1
    vals = np.empty(2 * nv * N)
    for k in range(2 * nv * N):
        s = (s * 6364136223846793005 + 1442695040888963407) & M64
        vals[k] = (s >> 11) / 9007199254740992.0 - 0.5
    return (vals[0::2] + 1j * vals[1::2]).reshape(nv, N).T


def power_rho(apply, N):
    """Power-iteration spectral-radius estimate with the device's schedule."""
    V = seeded_vectors(N)
    rho = 0.0
    for it in range(POWER_ITERS + 1):
        nrm = np.sqrt(np.sum(np.abs(V) ** 2, axis=0))
        if it > 0:
            rho = nrm.max()
            if it == POWER_ITERS:
                break
        V = apply(V * np.where(nrm > 0, 1.0 / np.where(nrm > 0, nrm, 1.0), 0.0))
    return rho


def coefficient_bound(rowptr, col, ratio, dinv):
    """(rho(K1), smax)."""
    N = len(rowptr) - 1
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    k1 = np.where(rows != col, ratio * dinv[col] / dinv[rows], 0.0)
    rho1 = power_rho(lambda V: spmm(rowptr, col, k1, V), N)
    return rho1, SREL / max(rho1, SREL)


def forward(p, F, Ef, rowptr, col, ratio, dinv):
    """Returns (M values on the pattern, cache for backward)."""
    N = F.shape[0]
    deg = np.diff(rowptr)
    rows = np.repeat(np.arange(N), deg)
    c = {"Z0": F @ p["W0"].T + p["b0"]}
    H = [relu(c["Z0"])]
    Zm, U, agg = [], [], []
    for l in range(GL):
        P = H[l] @ p[f"Wmh{l}"].T
        z = P[col] + Ef @ p[f"Wme{l}"].T + p[f"bm{l}"]
        a = np.zeros((N, GW))
        np.add.at(a, rows, relu(z))
        a /= np.maximum(deg, 1)[:, None]
        u = H[l] @ p[f"Wuh{l}"].T + a @ p[f"Wua{l}"].T + p[f"bu{l}"]
        Zm.append(z)
        agg.append(a)
        U.append(u)
        H.append(H[l] + relu(u))
    Zr = (H[GL] @ p["Wri"].T)[rows] + (H[GL] @ p["Wrj"].T)[col] + Ef @ p["Wrg"].T + p["br"]
    o = relu(Zr) @ p["Wo"].T + p["bo"]
    t = np.tanh(o)
    off = (rows != col).astype(float)
    rho1, smax = coefficient_bound(rowptr, col, ratio, dinv)
    cc = CMAX * (t[:, 0] + 1j * t[:, 1])
    ss = smax * (t[:, 2] + 0.5j * t[:, 3])
    m = ((1.0 - off) + cc - off * ss * ratio) * dinv[col]
    c.update(H=H, Zm=Zm, U=U, agg=agg, Zr=Zr, O=o, rows=rows, deg=deg, rho_ref=rho1, smax=smax)
    return m, c


def spmm(rowptr, col, val, X):
    N = len(rowptr) - 1
    Y = np.zeros((N,) + X.shape[1:], dtype=np.complex128)
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    np.add.at(Y, rows, val[:, None] * X[col] if X.ndim == 2 else val * X[col])
    return Y


def objective(A, rowptr, col, m, Z, b=None, x=None, lam=0.0):
    """L = |A M Z - Z|^2/(N p) + lam |M b - x|^2/|x|^2 and G = 2 dL/dconj(m)."""
    N, p = Z.shape
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    R = A @ spmm(rowptr, col, m, Z) - Z
    S = A.conj().T @ R
    L = np.sum(np.abs(R) ** 2) / (N * p)
    G = 2.0 / (N * p) * np.sum(S[rows] * Z[col].conj(), axis=1)
    if b is not None and lam > 0:
        rb = spmm(rowptr, col, m, b) - x
        xn = np.sum(np.abs(x) ** 2)
        L += lam * np.sum(np.abs(rb) ** 2) / xn
        G = G + 2.0 * lam / xn * rb[rows] * b[col].conj()
    return L, G


def backward(p, F, Ef, rowptr, col, ratio, dinv, c, G):
    """Gradients of the objective with respect to every parameter, from G
    (dL/dtheta = Re(conj(G) dm/dtheta) for every real parameter theta)."""
    N = F.shape[0]
    rows, deg = c["rows"], c["deg"]
    H, Zm, U, agg, Zr = c["H"], c["Zm"], c["U"], c["agg"], c["Zr"]
    g = {k: np.zeros_like(v) for k, v in p.items()}
    off = (rows != col).astype(float)
    t = G.conj() * dinv[col]
    u = t * ratio * off
    dO = np.stack([t.real, -t.imag, -u.real, u.imag], axis=1)
    dO = dO * np.array([CMAX, CMAX, c["smax"], 0.5 * c["smax"]]) * (1.0 - np.tanh(c["O"]) ** 2)
    Y = relu(Zr)
    g["Wo"] = dO.T @ Y
    g["bo"] = dO.sum(0)
    dZ = (dO @ p["Wo"]) * (Zr > 0)
    g["Wrg"] = dZ.T @ Ef
    g["br"] = dZ.sum(0)
    dP = np.zeros((N, GW))
    dQ = np.zeros((N, GW))
    np.add.at(dP, rows, dZ)
    np.add.at(dQ, col, dZ)
    g["Wri"] = dP.T @ H[GL]
    g["Wrj"] = dQ.T @ H[GL]
    dH = dP @ p["Wri"] + dQ @ p["Wrj"]
    for l in reversed(range(GL)):
        dU = dH * (U[l] > 0)
        g[f"Wuh{l}"] = dU.T @ H[l]
        g[f"bu{l}"] = dU.sum(0)
        g[f"Wua{l}"] = dU.T @ agg[l]
        dagg = dU @ p[f"Wua{l}"]
        dH = dH + dU @ p[f"Wuh{l}"]
        dZ = (dagg / np.maximum(deg, 1)[:, None])[rows] * (Zm[l] > 0)
        dP = np.zeros((N, GW))
        np.add.at(dP, col, dZ)
        g[f"Wme{l}"] = dZ.T @ Ef
        g[f"bm{l}"] = dZ.sum(0)
        g[f"Wmh{l}"] = dP.T @ H[l]
        dH = dH + dP @ p[f"Wmh{l}"]
    dZ0 = dH * (c["Z0"] > 0)
    g["W0"] = dZ0.T @ F
    g["b0"] = dZ0.sum(0)
    return g


def loss_and_grad(flat, F, Ef, rowptr, col, ratio, dinv, A, Z, b=None, x=None, lam=0.0):
    p = unpack(flat)
    m, c = forward(p, F, Ef, rowptr, col, ratio, dinv)
    L, G = objective(A, rowptr, col, m, Z, b, x, lam)
    return L, pack(backward(p, F, Ef, rowptr, col, ratio, dinv, c, G)), m
