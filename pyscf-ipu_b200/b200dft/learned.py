"""Learned initial guess: a message-passing network that predicts the initial density matrix.

The reference starts every SCF from MINAO (pyscf_utils/minao.py:5-123, dft.py:223).  This module
predicts D0 per atom-pair block from the geometry instead; the plain SCF still iterates every
molecule to the same convergence test, and ``RKSEngine.run_converged(fallback=...)`` restarts a
molecule from MINAO when its DIIS error rises.  Architecture (SchNet-style continuous-filter
message passing, feature size 128, 4 layers, 32 Gaussians on 0-5 A; hidden widths HL (layers,
site head) and HR (pair head): 384 / 576 give 0.97M parameters, 256 / 512 0.73M):

  h^0_a = E[type_a];  phi_p = rbf(r_p) Wf + bf;  m_a = sum_{p -> a} phi_p * h_src
  h^t   = h^{t-1} + silu(m Wa + ba) Wb + bb                                   (t = 1..4)
  pair a<b within 5 A: z = W3 silu(W2 silu(W1 [h_a, h_b, rbf_ab] + b1) + b2) + b3   (16 scalars)
  site a:              y = V2 silu(V1 h_a + c1) + c2                               (4 scalars)
  blocks: ss = z0..3, s_a p_b = z4,5 u, p_a s_b = z6,7 u, p_a p_b = z8 u u^T + z9 (I - u u^T);
          onsite ss = y0..2, pp = y3 I, plus neighbour sums s_a p_a += z10,11 u, p_a p_a += z12 u u^T,
          s_b p_b -= z13,14 u, p_b p_b += z15 u u^T   (u = unit vector a -> b: blocks rotate with
          the molecule; D is mirrored to be symmetric)

Training and inference run on the GPU through this project's kernels (csrc/learned.cu): every
matrix product rounds its inputs to bfloat16 and accumulates in float32; master weights and Adam
state are float32.  Training targets are converged densities produced by the SCF engine itself.
"""
import ctypes
import numpy as np
import torch

from ._lib import lib, check, ptr, stream_handle

F, R, L = 128, 32, 4
HL, HR = 384, 576                       # hidden widths of new networks (a weights file records its own)
NT = 5
TYPE = {1: 0, 6: 1, 7: 2, 8: 3, 9: 4}
RC = 5.0 / 0.52917721092                # 5 Angstrom in Bohr

_P, _I, _L, _F = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
_SIG = {
    "b2_nn_gemm": [_I, _I, _I, _P, _L, _L, _P, _L, _L, _P, _L, _P, _F, _I, _P],
    "b2_nn_colsum": [_I, _I, _P, _L, _P, _I, _P],
    "b2_nn_silu": [_L, _P, _P, _P],
    "b2_nn_silu_bwd": [_L, _P, _P, _P, _P],
    "b2_nn_rbf": [_L, _I, _F, _P, _P, _P],
    "b2_nn_message": [_I, _I, _P, _P, _P, _P, _P, _I, _P],
    "b2_nn_pairmul": [_L, _I, _P, _P, _P, _P, _P, _P],
    "b2_nn_gather": [_L, _I, _I, _P, _P, _P, _P, _P, _P],
    "b2_nn_scatter": [_L, _I, _I, _P, _P, _P, _P, _P],
    "b2_nn_embed": [_I, _I, _P, _P, _P, _P],
    "b2_nn_embed_bwd": [_I, _I, _P, _P, _P, _P],
    "b2_nn_assemble": [_L, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _L, _P, _P, _P, _P, _P, _P],
    "b2_nn_adam": [_L, _P, _P, _P, _P, _F, _F, _F, _F, _I, _F, _P],
}
_bound = False


def _lib():
    global _bound
    L_ = lib()
    if not _bound:
        for n, a in _SIG.items():
            f = getattr(L_, n)
            f.argtypes = a
            f.restype = ctypes.c_int
        _bound = True
    return L_


def layout(hl=HL, hr=HR):
    HL, HR = hl, hr
    shapes = [("E", (NT, F))]
    for t in range(L):
        shapes += [(f"Wf{t}", (R, F)), (f"bf{t}", (F,)), (f"Wa{t}", (F, HL)), (f"ba{t}", (HL,)),
                   (f"Wb{t}", (HL, F)), (f"bb{t}", (F,))]
    shapes += [("W1", (2 * F + R, HR)), ("b1", (HR,)), ("W2", (HR, HR)), ("b2", (HR,)),
               ("W3", (HR, 16)), ("b3", (16,)), ("V1", (F, HL)), ("c1", (HL,)), ("V2", (HL, 4)), ("c2", (4,))]
    return shapes


def init_params_np(seed=0, hl=HL, hr=HR):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shp in layout(hl, hr):
        if name[0] in "bc":
            p[name] = np.zeros(shp)
        elif name == "E":
            p[name] = rng.normal(size=shp)
        else:
            p[name] = rng.normal(size=shp) * np.sqrt(1.0 / shp[0])
    for t in range(L):
        p[f"Wb{t}"] *= 0.1
    return p


class Batch:
    """Graph of a list of molecules, built on ``device`` (edge and pair lists stay there)."""

    def __init__(self, mols, device="cuda", mat_off=None, nao=None):
        # all molecules at once on a padded (molecule, atom, atom) grid; edge order per molecule
        # is by receiving atom then sending atom, pair order by (a, b) with a < b
        nat = np.array([m.natm for m in mols], np.int64)
        self.n_atoms = [int(n) for n in nat]
        nm, amax = len(mols), int(nat.max()) if len(mols) else 0
        valid_h = np.arange(amax)[None, :] < nat[:, None]
        Ch = np.zeros((nm, amax, 3))
        Zh = np.zeros((nm, amax), np.int64)
        if nm:
            Ch[valid_h] = np.concatenate([m.coords for m in mols])
            Zh[valid_h] = np.concatenate([m.charges for m in mols])
        dev = torch.device(device)
        base_h = (np.concatenate([[0], np.cumsum(nat)[:-1]]).astype(np.int64) if nm else np.zeros(0, np.int64))
        C = torch.from_numpy(Ch).to(dev)
        valid = torch.from_numpy(valid_h).to(dev)
        base = torch.from_numpy(base_h).to(dev)
        d = torch.sqrt(((C[:, :, None] - C[:, None]) ** 2).sum(-1))
        close = (d < RC) & valid[:, :, None] & valid[:, None, :]
        edge = close & ~torch.eye(amax, dtype=torch.bool, device=dev)[None]
        em, et, es = torch.nonzero(edge.transpose(1, 2), as_tuple=True)   # (molecule, receiver, sender)
        i32, f32 = torch.int32, torch.float32
        src, dst, rr = (es + base[em]).to(i32), (et + base[em]).to(i32), d[em, es, et].to(f32)
        pm, a, b = torch.nonzero(torch.triu(close, 1) if amax else close, as_tuple=True)
        pa, pb, pr = (a + base[pm]).to(i32), (b + base[pm]).to(i32), d[pm, a, b].to(f32)
        u = C[pm, b] - C[pm, a]
        pu = (u / torch.clamp(torch.linalg.norm(u, dim=1, keepdim=True), min=1e-30)).to(f32).reshape(-1)
        zf = Zh[valid_h]
        self.A, self.P, self.Pr = int(len(zf)), int(src.numel()), int(pa.numel())
        mol_of = np.repeat(np.arange(nm), nat)
        width = np.where(Zh <= 2, 1, 5) * valid_h
        ao0 = (np.cumsum(width, 1) - width)[valid_h]
        tmap = np.zeros(max(TYPE) + 1 if TYPE else 1, np.int32)
        for zz, tt in TYPE.items():
            tmap[zz] = tt
        types = tmap[zf].astype(np.int32)
        heavy = (zf > 2).astype(np.int64)
        atoms = np.stack([mol_of, ao0, heavy, np.zeros(self.A, np.int64)], 1).astype(np.int32)
        cnt = torch.bincount(dst.to(torch.int64), minlength=self.A)
        ptr_ = torch.zeros(self.A + 1, dtype=torch.int64, device=dev)
        ptr_[1:] = torch.cumsum(cnt, 0)
        naos = np.array([m.nao for m in mols], np.int32)
        if mat_off is None:
            mat_off = np.concatenate([[0], np.cumsum(naos.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
        self.mat_off = np.ascontiguousarray(mat_off, np.int64)
        self.nao = np.ascontiguousarray(naos if nao is None else nao, np.int32)
        self.n_mat = int(self.mat_off[-1] + self.nao[-1].astype(np.int64) ** 2) if len(mols) else 0
        self.nent = self.n_mat                 # the loss averages over every matrix entry
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        self.h2d_bytes = int(Ch.nbytes + valid_h.nbytes + base_h.nbytes + types.nbytes + atoms.nbytes +
                             self.mat_off.nbytes + self.nao.nbytes)     # host -> device copies
        self.d = {"src": src, "dst": dst, "r": rr, "pa": pa, "pb": pb, "pr": pr, "pu": pu.contiguous(),
                  "types": t(types), "ptr": ptr_.to(i32), "atoms": t(atoms), "mat_off": t(self.mat_off),
                  "nao": t(self.nao)}


class GuessNet:
    """Parameters, forward/backward through the CUDA kernels, Adam, D0 prediction."""

    def __init__(self, seed=0, device="cuda", bf16=True, tensor_cores=True, hl=HL, hr=HR):
        self.device = torch.device(device)
        self.hl, self.hr = hl, hr
        # 0: float32 SIMT (exact, for checks); 1: bf16-rounded SIMT; 2: bf16 tcgen05 tensor cores
        self.bf16 = (2 if tensor_cores else 1) if bf16 else 0
        self.shapes = layout(hl, hr)
        self.offsets = {}
        o = 0
        for n, s in self.shapes:
            self.offsets[n] = (o, s)
            o += int(np.prod(s))
        self.n_params = o
        p = init_params_np(seed, hl, hr)
        flat = np.concatenate([p[n].reshape(-1) for n, _ in self.shapes]).astype(np.float32)
        self.params = torch.from_numpy(flat).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0

    def P(self, name, grad=False):
        o, s = self.offsets[name]
        t = self.grads if grad else self.params
        return t[o:o + int(np.prod(s))].view(*s)

    # ---- primitives ------------------------------------------------------------------------
    def _mm(self, X, W, bias=None, out=None, beta=0.0):
        """out = X @ W (+ bias), X (M,K) row-major, W (K,N) row-major"""
        M, K = X.shape
        N = W.shape[1]
        if out is None:
            out = torch.empty((M, N), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_gemm(M, N, K, ptr(X), K, 1, ptr(W), N, 1, ptr(out), N, ptr(bias), beta, self.bf16,
                                stream_handle()), "b2_nn_gemm")
        return out

    def _mm_tn(self, X, dY, out, beta=1.0):
        """out (K,N) (+)= X^T @ dY   (X (M,K), dY (M,N))"""
        M, K = X.shape
        N = dY.shape[1]
        check(_lib().b2_nn_gemm(K, N, M, ptr(X), 1, K, ptr(dY), N, 1, ptr(out), N, None, beta, self.bf16,
                                stream_handle()), "b2_nn_gemm")

    def _mm_nt(self, dY, W, out=None, beta=0.0):
        """out (M,K) = dY @ W^T   (dY (M,N), W (K,N))"""
        M, N = dY.shape
        K = W.shape[0]
        if out is None:
            out = torch.empty((M, K), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_gemm(M, K, N, ptr(dY), N, 1, ptr(W), 1, N, ptr(out), K, None, beta, self.bf16,
                                stream_handle()), "b2_nn_gemm")
        return out

    def _colsum(self, X, out):
        check(_lib().b2_nn_colsum(X.shape[0], X.shape[1], ptr(X), X.shape[1], ptr(out), 1, stream_handle()),
              "b2_nn_colsum")

    def _silu(self, x):
        y = torch.empty_like(x)
        check(_lib().b2_nn_silu(x.numel(), ptr(x), ptr(y), stream_handle()), "b2_nn_silu")
        return y

    def _silu_bwd(self, x, dy):
        dx = torch.empty_like(x)
        check(_lib().b2_nn_silu_bwd(x.numel(), ptr(x), ptr(dy), ptr(dx), stream_handle()), "b2_nn_silu_bwd")
        return dx

    def _rbf(self, r):
        out = torch.empty((r.numel(), R), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_rbf(r.numel(), R, float(RC), ptr(r), ptr(out), stream_handle()), "b2_nn_rbf")
        return out

    # ---- model -----------------------------------------------------------------------------
    def forward(self, B):
        d = B.d
        c = {}
        h = torch.empty((B.A, F), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_embed(B.A, F, ptr(d["types"]), ptr(self.P("E")), ptr(h), stream_handle()), "embed")
        rb = self._rbf(d["r"])
        c["rb"], c["h"] = rb, [h]
        c["layers"] = []
        for t in range(L):
            phi = self._mm(rb, self.P(f"Wf{t}"), self.P(f"bf{t}"))
            m = torch.empty((B.A, F), dtype=torch.float32, device=self.device)
            check(_lib().b2_nn_message(B.A, F, ptr(d["ptr"]), ptr(d["src"]), ptr(phi), ptr(h), ptr(m), 0,
                                       stream_handle()), "message")
            a1 = self._mm(m, self.P(f"Wa{t}"), self.P(f"ba{t}"))
            s1 = self._silu(a1)
            hn = h.clone()
            self._mm(s1, self.P(f"Wb{t}"), self.P(f"bb{t}"), out=hn, beta=1.0)
            c["layers"].append((phi, m, a1, s1))
            h = hn
            c["h"].append(h)
        rbp = self._rbf(d["pr"])
        x = torch.empty((B.Pr, 2 * F + R), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_gather(B.Pr, F, R, ptr(d["pa"]), ptr(d["pb"]), ptr(h), ptr(rbp), ptr(x),
                                  stream_handle()), "gather")
        q1 = self._mm(x, self.P("W1"), self.P("b1"))
        u1 = self._silu(q1)
        q2 = self._mm(u1, self.P("W2"), self.P("b2"))
        u2 = self._silu(q2)
        z = self._mm(u2, self.P("W3"), self.P("b3"))
        v1 = self._mm(h, self.P("V1"), self.P("c1"))
        w1 = self._silu(v1)
        y = self._mm(w1, self.P("V2"), self.P("c2"))
        c.update(x=x, q1=q1, u1=u1, q2=q2, u2=u2, v1=v1, w1=w1)
        return z, y, c

    def assemble(self, B, z, y, D, Dt=None):
        """D (zeroed here) <- predicted densities (B's matrix layout); with targets also return the
        mean squared error over all entries and dL/dz, dL/dy"""
        D.zero_()
        dz = torch.zeros_like(z) if Dt is not None else None
        dy = torch.zeros_like(y) if Dt is not None else None
        Rb = torch.empty_like(D) if Dt is not None else None
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        d = B.d
        check(_lib().b2_nn_assemble(B.Pr, ptr(d["pa"]), ptr(d["pb"]), ptr(d["pu"]), B.A, ptr(d["atoms"]),
                                    ptr(d["mat_off"]), ptr(d["nao"]), ptr(z), ptr(y), ptr(D), B.n_mat, ptr(Dt),
                                    ptr(Rb), ptr(dz), ptr(dy), ptr(loss), stream_handle()), "assemble")
        return loss, dz, dy

    def backward(self, B, c, dz, dy):
        d = B.d
        self.grads.zero_()
        G = lambda n: self.P(n, grad=True)
        self._mm_tn(c["u2"], dz, G("W3")); self._colsum(dz, G("b3"))
        du2 = self._mm_nt(dz, self.P("W3"))
        dq2 = self._silu_bwd(c["q2"], du2)
        self._mm_tn(c["u1"], dq2, G("W2")); self._colsum(dq2, G("b2"))
        du1 = self._mm_nt(dq2, self.P("W2"))
        dq1 = self._silu_bwd(c["q1"], du1)
        self._mm_tn(c["x"], dq1, G("W1")); self._colsum(dq1, G("b1"))
        dx = self._mm_nt(dq1, self.P("W1"))
        h = c["h"][-1]
        dh = torch.zeros((B.A, F), dtype=torch.float32, device=self.device)
        check(_lib().b2_nn_scatter(B.Pr, F, R, ptr(d["pa"]), ptr(d["pb"]), ptr(dx), ptr(dh), stream_handle()),
              "scatter")
        self._mm_tn(c["w1"], dy, G("V2")); self._colsum(dy, G("c2"))
        dw1 = self._mm_nt(dy, self.P("V2"))
        dv1 = self._silu_bwd(c["v1"], dw1)
        self._mm_tn(h, dv1, G("V1")); self._colsum(dv1, G("c1"))
        self._mm_nt(dv1, self.P("V1"), out=dh, beta=1.0)
        rb = c["rb"]
        for t in reversed(range(L)):
            phi, m, a1, s1 = c["layers"][t]
            hp = c["h"][t]
            self._mm_tn(s1, dh, G(f"Wb{t}")); self._colsum(dh, G(f"bb{t}"))
            ds1 = self._mm_nt(dh, self.P(f"Wb{t}"))
            da1 = self._silu_bwd(a1, ds1)
            self._mm_tn(m, da1, G(f"Wa{t}")); self._colsum(da1, G(f"ba{t}"))
            dm = self._mm_nt(da1, self.P(f"Wa{t}"))
            dphi = torch.empty_like(phi)
            check(_lib().b2_nn_pairmul(B.P, F, ptr(d["src"]), ptr(d["dst"]), ptr(dm), ptr(hp), ptr(dphi),
                                       stream_handle()), "pairmul")
            self._mm_tn(rb, dphi, G(f"Wf{t}")); self._colsum(dphi, G(f"bf{t}"))
            # dh_prev = dh + sum_{p: src=a} dm[dst] phi_p = dh + message(phi, dm) (symmetric graph)
            check(_lib().b2_nn_message(B.A, F, ptr(d["ptr"]), ptr(d["src"]), ptr(phi), ptr(dm), ptr(dh), 1,
                                       stream_handle()), "message_bwd")
        check(_lib().b2_nn_embed_bwd(B.A, F, ptr(d["types"]), ptr(dh), ptr(G("E")), stream_handle()), "embed_bwd")
        return self.grads

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.step_count += 1
        check(_lib().b2_nn_adam(self.n_params, ptr(self.params), ptr(self.grads), ptr(self.m), ptr(self.v),
                                lr, b1, b2, eps, self.step_count, wd, stream_handle()), "adam")

    def train_step(self, B, Dt, lr=1e-3):
        z, y, c = self.forward(B)
        D = torch.zeros(B.n_mat, dtype=torch.float64, device=self.device)
        loss, dz, dy = self.assemble(B, z, y, D, Dt)
        self.backward(B, c, dz, dy)
        self.adam(lr)
        return loss

    def predict(self, B, D):
        """write the predicted initial densities into D (B's matrix layout)"""
        z, y, _ = self.forward(B)
        self.assemble(B, z, y, D)
        return D
