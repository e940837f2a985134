"""numpy reference of the learned initial-guess network (test infrastructure).

Checks the GPU forward/backward kernels of b200dft.learned.  The reference has no such
network (it starts every SCF from MINAO, minao.py:5-123); the architecture is this
project's (SchNet-style continuous-filter message passing, as in the reference's consumer
model schnet_9m/model.py:76-140, scaled to the density-matrix task):

  h_a^0     = E[type_a]                                              (F)
  rbf_p     = exp(-g (r_p - mu_k)^2) fc(r_p)                          (R)  directed pairs p = (src -> dst)
  phi_p^t   = rbf_p Wf_t + bf_t                                       (F)
  m_a^t     = sum_{p: dst = a} phi_p^t * h_src^{t-1}                   (F)
  h^t       = h^{t-1} + silu(m^t Wa_t + ba_t) Wb_t + bb_t              (F -> HL -> F)
  pair a<b  : x = [h_a, h_b, rbf_ab], z = W3 silu(W2 silu(W1 x + b1) + b2) + b3   (16 scalars)
  site a    : y = V2 silu(V1 h_a + c1) + c2                            (4 scalars)
Blocks are built from the scalars and u = (R_b - R_a)/|R_b - R_a| so that they rotate with the
molecule: ss = z0..z3, s_a p_b = z4/z5 u, p_a s_b = z6/z7 u, p_a p_b = z8 u u^T + z9 (I - u u^T);
onsite ss = y0, y1, y2 and pp = y3 I plus, summed over the neighbours b of a, s_a p_a += z10/z11 u
and p_a p_a += z12 u u^T (and for b: s_b p_b -= z13/z14 u, p_b p_b += z15 u u^T).  Every block is
mirrored (D symmetric).  The loss is the mean squared error against the converged density over
all entries of each molecule's matrix.
"""
import numpy as np

F, R, HL, HR, L = 128, 32, 256, 512, 4
NT = 5                                  # H, C, N, O, F
TYPE = {1: 0, 6: 1, 7: 2, 8: 3, 9: 4}
RC = 5.0 / 0.52917721092                # 5 Angstrom cutoff in Bohr


def layout():
    """parameter name -> shape, in the order of the flat parameter vector"""
    shapes = [("E", (NT, F))]
    for t in range(L):
        shapes += [(f"Wf{t}", (R, F)), (f"bf{t}", (F,)), (f"Wa{t}", (F, HL)), (f"ba{t}", (HL,)),
                   (f"Wb{t}", (HL, F)), (f"bb{t}", (F,))]
    shapes += [("W1", (2 * F + R, HR)), ("b1", (HR,)), ("W2", (HR, HR)), ("b2", (HR,)),
               ("W3", (HR, 16)), ("b3", (16,)), ("V1", (F, HL)), ("c1", (HL,)), ("V2", (HL, 4)), ("c2", (4,))]
    return shapes


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shp in layout():
        if name[0] in "b" or name[0] == "c":
            p[name] = np.zeros(shp)
        elif name == "E":
            p[name] = rng.normal(size=shp)
        else:
            p[name] = rng.normal(size=shp) * np.sqrt(1.0 / shp[0])
    for t in range(L):
        p[f"Wb{t}"] *= 0.1
    return p


def rbf(r):
    mu = np.linspace(0, RC, R)
    g = 1.0 / (2 * (RC / (R - 1)) ** 2)
    fc = np.where(r < RC, 0.5 * (np.cos(np.pi * r / RC) + 1), 0.0)
    return np.exp(-g * (r[:, None] - mu[None, :]) ** 2) * fc[:, None]


def silu(x):
    return x / (1 + np.exp(-x))


def dsilu(x):
    s = 1 / (1 + np.exp(-x))
    return s * (1 + x * (1 - s))


def graph(charges, coords):
    """directed pairs within the cutoff (src, dst), readout pairs a<b within the cutoff"""
    n = len(charges)
    d = np.sqrt(((coords[:, None] - coords[None]) ** 2).sum(-1))
    src, dst = np.where((d < RC) & ~np.eye(n, dtype=bool))
    a, b = np.where(np.triu(d < RC, 1))
    return src, dst, d[src, dst], a, b, d[a, b]


def forward(p, charges, coords, cache=False):
    types = np.array([TYPE[int(z)] for z in charges])
    src, dst, r, pa, pb, pr = graph(charges, coords)
    h = p["E"][types].copy()
    rb = rbf(r)
    C = {"types": types, "src": src, "dst": dst, "rb": rb, "hs": [h.copy()], "layers": []}
    for t in range(L):
        phi = rb @ p[f"Wf{t}"] + p[f"bf{t}"]
        m = np.zeros_like(h)
        np.add.at(m, dst, phi * h[src])
        a1 = m @ p[f"Wa{t}"] + p[f"ba{t}"]
        s1 = silu(a1)
        h = h + s1 @ p[f"Wb{t}"] + p[f"bb{t}"]
        C["layers"].append((phi, m, a1, s1))
        C["hs"].append(h.copy())
    rbp = rbf(pr)
    x = np.concatenate([h[pa], h[pb], rbp], 1)
    q1 = x @ p["W1"] + p["b1"]
    u1 = silu(q1)
    q2 = u1 @ p["W2"] + p["b2"]
    u2 = silu(q2)
    z = u2 @ p["W3"] + p["b3"]
    v1 = h @ p["V1"] + p["c1"]
    w1 = silu(v1)
    y = w1 @ p["V2"] + p["c2"]
    C.update(pa=pa, pb=pb, x=x, q1=q1, u1=u1, q2=q2, u2=u2, v1=v1, w1=w1, h=h)
    return (z, y, C) if cache else (z, y)


def ao_offsets(charges):
    off, o = [], 0
    for zc in charges:
        off.append(o)
        o += 1 if zc <= 2 else 5
    return np.array(off), o


def visits(charges, coords, pa, pb):
    """linear structure of the assembly: list of (row, col, kind, index, scalar, coef) with
    kind 'z' (pair scalars) or 'y' (site scalars); D[row, col] = sum coef * scalar"""
    off, n = ao_offsets(charges)
    heavy = [zc > 2 for zc in charges]
    out = []
    def sym(r, c, kind, idx, k, coef):
        out.append((r, c, kind, idx, k, coef))
        if r != c:
            out.append((c, r, kind, idx, k, coef))
    for a in range(len(charges)):
        o = off[a]
        sym(o, o, "y", a, 0, 1.0)
        if heavy[a]:
            sym(o, o + 1, "y", a, 1, 1.0)
            sym(o + 1, o + 1, "y", a, 2, 1.0)
            for c in range(3):
                sym(o + 2 + c, o + 2 + c, "y", a, 3, 1.0)
    for k, (a, b) in enumerate(zip(pa, pb)):
        u = coords[b] - coords[a]
        u = u / np.linalg.norm(u)
        oa, ob = off[a], off[b]
        sa = [oa] + ([oa + 1] if heavy[a] else [])
        sb = [ob] + ([ob + 1] if heavy[b] else [])
        for i, ia in enumerate(sa):
            for j, jb in enumerate(sb):
                sym(ia, jb, "z", k, 2 * i + j, 1.0)
        if heavy[b]:
            for i, ia in enumerate(sa):
                for d in range(3):
                    sym(ia, ob + 2 + d, "z", k, 4 + i, u[d])
        if heavy[a]:
            for j, jb in enumerate(sb):
                for c in range(3):
                    sym(oa + 2 + c, jb, "z", k, 6 + j, u[c])
        if heavy[a] and heavy[b]:
            for c in range(3):
                for d in range(3):
                    sym(oa + 2 + c, ob + 2 + d, "z", k, 8, u[c] * u[d])
                    sym(oa + 2 + c, ob + 2 + d, "z", k, 9, (c == d) - u[c] * u[d])
        if heavy[a]:
            for i, ia in enumerate(sa):
                for c in range(3):
                    sym(ia, oa + 2 + c, "z", k, 10 + i, u[c])
            for c in range(3):
                for d in range(3):
                    out.append((oa + 2 + c, oa + 2 + d, "z", k, 12, u[c] * u[d]))
        if heavy[b]:
            for j, jb in enumerate(sb):
                for c in range(3):
                    sym(jb, ob + 2 + c, "z", k, 13 + j, -u[c])
            for c in range(3):
                for d in range(3):
                    out.append((ob + 2 + c, ob + 2 + d, "z", k, 15, u[c] * u[d]))
    return out, n


def assemble(z, y, charges, coords, pa, pb):
    """predicted density matrix (full, symmetric)"""
    vis, n = visits(charges, coords, pa, pb)
    D = np.zeros((n, n))
    for r, c, kind, idx, k, coef in vis:
        D[r, c] += coef * (z[idx, k] if kind == "z" else y[idx, k])
    return D


def loss(z, y, charges, coords, pa, pb, Dt):
    Dp = assemble(z, y, charges, coords, pa, pb)
    return float(((Dp - Dt) ** 2).mean()), Dp


def grad_scalars(z, y, charges, coords, pa, pb, Dt):
    """dL/dz, dL/dy (the assembly is linear in the scalars)"""
    Dp = assemble(z, y, charges, coords, pa, pb)
    Rm = 2 * (Dp - Dt) / Dp.size
    vis, _ = visits(charges, coords, pa, pb)
    gz = np.zeros_like(z)
    gy = np.zeros_like(y)
    for r, c, kind, idx, k, coef in vis:
        if kind == "z":
            gz[idx, k] += coef * Rm[r, c]
        else:
            gy[idx, k] += coef * Rm[r, c]
    return gz, gy


def backward(p, charges, coords, Dt):
    """loss and gradients of every parameter (analytic, float64)"""
    z, y, C = forward(p, charges, coords, cache=True)
    L0, _ = loss(z, y, charges, coords, C["pa"], C["pb"], Dt)
    gz, gy = grad_scalars(z, y, charges, coords, C["pa"], C["pb"], Dt)
    g = {k: np.zeros_like(v) for k, v in p.items()}
    # readout
    g["W3"] = C["u2"].T @ gz
    g["b3"] = gz.sum(0)
    du2 = gz @ p["W3"].T
    dq2 = du2 * dsilu(C["q2"])
    g["W2"] = C["u1"].T @ dq2
    g["b2"] = dq2.sum(0)
    du1 = dq2 @ p["W2"].T
    dq1 = du1 * dsilu(C["q1"])
    g["W1"] = C["x"].T @ dq1
    g["b1"] = dq1.sum(0)
    dx = dq1 @ p["W1"].T
    h = C["h"]
    dh = np.zeros_like(h)
    np.add.at(dh, C["pa"], dx[:, :F])
    np.add.at(dh, C["pb"], dx[:, F:2 * F])
    g["V2"] = C["w1"].T @ gy
    g["c2"] = gy.sum(0)
    dw1 = gy @ p["V2"].T
    dv1 = dw1 * dsilu(C["v1"])
    g["V1"] = h.T @ dv1
    g["c1"] = dv1.sum(0)
    dh += dv1 @ p["V1"].T
    # message-passing layers in reverse
    src, dst, rb = C["src"], C["dst"], C["rb"]
    for t in reversed(range(L)):
        phi, m, a1, s1 = C["layers"][t]
        hp = C["hs"][t]
        g[f"Wb{t}"] = s1.T @ dh
        g[f"bb{t}"] = dh.sum(0)
        ds1 = dh @ p[f"Wb{t}"].T
        da1 = ds1 * dsilu(a1)
        g[f"Wa{t}"] = m.T @ da1
        g[f"ba{t}"] = da1.sum(0)
        dm = da1 @ p[f"Wa{t}"].T
        dphi = dm[dst] * hp[src]
        g[f"Wf{t}"] = rb.T @ dphi
        g[f"bf{t}"] = dphi.sum(0)
        dhp = dh.copy()
        np.add.at(dhp, src, dm[dst] * phi)
        dh = dhp
    np.add.at(g["E"], C["types"], dh)
    return L0, g
