"""Batched RKS engine on one B200: host setup + device SCF loop through the C ABI.

One ``RKSEngine`` holds a batch of molecules (one molecule for the drop-in entry points).
Host setup mirrors what the reference does on the host with PySCF before its jitted SCF
(dft.py:197-234, nanoDFT.py:208-257): molecule/basis (``Mole``), grid (``Grids``),
one-electron matrices (``int1e``), L = inv(cholesky(S)) and the MINAO-style guess.  All
arrays are then packed per molecule (offsets from the plan) into device buffers, and the
SCF loop runs entirely on the device: ERIs once, then per iteration Fock+DIIS,
orthogonalised eigensolve + density, XC and J/K, energies (nanoDFT.py:40-102).
"""
import ctypes
import numpy as np
import torch

from ._lib import lib, check, ptr, stream_handle, B200DFTError
from .constants import HYB_B3LYP
from .grids import Grids
from .guess import minao
from .int1e import int1e

NMO = 72     # mo_energy row stride used by the device kernels


class Plan:
    """Owner of a ``b2_plan_t`` built from the molecules' libcint arrays."""

    def __init__(self, mols):
        self.mols = list(mols)
        nmol = len(self.mols)
        natm = np.array([m.natm for m in self.mols], np.int32)
        nbas = np.array([m.nbas for m in self.mols], np.int32)
        atm = np.ascontiguousarray(np.concatenate([m._atm for m in self.mols]), dtype=np.int32)
        bas = np.ascontiguousarray(np.concatenate([m._bas for m in self.mols]), dtype=np.int32)
        env = np.ascontiguousarray(np.concatenate([m._env for m in self.mols]), dtype=np.float64)
        env_off = np.cumsum([0] + [len(m._env) for m in self.mols[:-1]]).astype(np.int64)
        h = ctypes.c_void_p()
        check(lib().b2_plan_create(nmol, ptr(natm), ptr(nbas), ptr(atm), ptr(bas), ptr(env),
                                   ptr(env_off), ctypes.byref(h)), "b2_plan_create")
        self.h = h
        info = np.zeros(8, np.int64)
        check(lib().b2_plan_info(h, ptr(info)), "b2_plan_info")
        self.n_eri, self.n_mat, self.nmol, self.max_nao = (int(x) for x in info[:4])
        self.n_rows, self.n_sp = int(info[4]), int(info[5])
        self.eri_off = np.zeros(nmol, np.int64)
        self.mat_off = np.zeros(nmol, np.int64)
        self.nao = np.zeros(nmol, np.int32)
        self.nocc = np.zeros(nmol, np.int32)
        check(lib().b2_plan_offsets(h, ptr(self.eri_off), ptr(self.mat_off), ptr(self.nao),
                                    ptr(self.nocc)), "b2_plan_offsets")
        self.grid_off = None

    def set_grid(self, npoints):
        goff = np.concatenate([[0], np.cumsum(npoints)]).astype(np.int64)
        check(lib().b2_grid_set(self.h, ptr(goff)), "b2_grid_set")
        npts, nao = ctypes.c_int64(), ctypes.c_int64()
        check(lib().b2_grid_info(self.h, ctypes.byref(npts), ctypes.byref(nao)), "b2_grid_info")
        self.grid_off = goff
        self.n_points, self.n_ao = npts.value, nao.value
        self.ao_off = np.zeros(self.nmol, np.int64)
        check(lib().b2_grid_ao_offsets(self.h, ptr(self.ao_off)), "b2_grid_ao_offsets")

    def set_jk_chunk(self, elems):
        check(lib().b2_plan_set_jk_chunk(self.h, int(elems)), "b2_plan_set_jk_chunk")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().b2_plan_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # matrices ------------------------------------------------------------------------
    def pack(self, mats):
        out = np.zeros(self.n_mat, np.float64)
        for m, a in enumerate(mats):
            n = self.nao[m]
            out[self.mat_off[m]:self.mat_off[m] + n * n] = np.asarray(a, np.float64).reshape(-1)
        return out

    def unpack(self, flat, m):
        n = int(self.nao[m])
        o = int(self.mat_off[m])
        return flat[o:o + n * n].reshape(n, n)


def _require_cuda():
    if not torch.cuda.is_available():
        raise B200DFTError("no CUDA device: the b200dft engine runs on the GPU only (no CPU fallback)")


class HostSetup:
    """Per-molecule host inputs (the reference's PySCF-side setup)."""

    def __init__(self, mol, level=0, grid=None, D0=None):
        self.mol = mol
        S, T, V = int1e(mol)
        self.S, self.T, self.V = S, T, V
        self.Hcore = T + V
        self.L_inv = np.linalg.inv(np.linalg.cholesky(S))
        if grid is None:
            grid = Grids(mol, level).build()
        self.coords = np.ascontiguousarray(grid.coords, np.float64)
        self.weights = np.ascontiguousarray(grid.weights, np.float64)
        self.D0 = minao(mol) if D0 is None else np.asarray(D0, np.float64)
        self.E_nuc = mol.energy_nuc()


class RKSEngine:
    """Device SCF for a batch of molecules.

    precision: "fp64" (plain: FP64 ERIs, J/K and grid path) or "mixed" (FP32 ERIs, J/K and
    grid path; FP64 Fock/DIIS/eigensolve/energies).
    """

    def __init__(self, mols, level=0, precision="fp64", setups=None, device=None, jk_chunk=None):
        _require_cuda()
        self.mols = list(mols)
        self.precision = precision
        self.prec = 64 if precision == "fp64" else 32
        self.device = torch.device(device or "cuda")
        self.setups = setups or [HostSetup(m, level) for m in self.mols]
        self.plan = Plan(self.mols)
        if jk_chunk:
            self.plan.set_jk_chunk(jk_chunk)
        P = self.plan
        self.plan.set_grid([len(s.weights) for s in self.setups])
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        rdt = torch.float64 if self.prec == 64 else torch.float32
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.S = t(P.pack([s.S for s in self.setups]))
        self.Hcore = t(P.pack([s.Hcore for s in self.setups]))
        self.Linv = t(P.pack([s.L_inv for s in self.setups]))
        self.D0 = t(P.pack([s.D0 for s in self.setups]))
        self.coords = t(np.concatenate([s.coords for s in self.setups]).reshape(-1))
        self.weights = t(np.concatenate([s.weights for s in self.setups]))
        self.enuc = torch.tensor([s.E_nuc for s in self.setups], **f64)
        nm, nmat = P.nmol, P.n_mat
        self.eri = torch.empty(P.n_eri, dtype=rdt, device=dev)
        self.ao = torch.empty(max(1, P.n_ao), dtype=rdt, device=dev)
        z = lambda n: torch.zeros(n, **f64)
        self.D, self.J, self.K, self.Vxc = z(nmat), z(nmat), z(nmat), z(nmat)
        self.H, self.diffJK = z(nmat), z(nmat)
        self.ring_err, self.ring_h = z(9 * nmat), z(9 * nmat)
        self.bmat = z(100 * nm)
        self.diis_err = z(nm)
        self.exc = z(nm)
        self.energy = z(5 * nm)
        self.mo_energy = z(NMO * nm)
        self.C = z(nmat)
        self.iter = torch.zeros(nm, dtype=torch.int32, device=dev)
        self.active = torch.ones(nm, dtype=torch.int32, device=dev)
        self.sweeps = torch.zeros(nm, dtype=torch.int32, device=dev)
        self._eri_done = False
        self._ao_done = False

    # --- kernels -----------------------------------------------------------------------
    def compute_eri(self, stream=None):
        check(lib().b2_eri_s8(self.plan.h, self.prec, ptr(self.eri), stream_handle(stream)), "b2_eri_s8")
        self._eri_done = True

    def compute_ao(self, stream=None):
        check(lib().b2_ao_eval(self.plan.h, self.prec, ptr(self.coords), ptr(self.ao),
                               stream_handle(stream)), "b2_ao_eval")
        self._ao_done = True

    def jk(self, D=None, stream=None):
        D = self.D if D is None else D
        check(lib().b2_jk_s8(self.plan.h, self.prec, ptr(self.eri), ptr(D), ptr(self.J), ptr(self.K),
                             stream_handle(stream)), "b2_jk_s8")

    def xc(self, D=None, stream=None):
        D = self.D if D is None else D
        check(lib().b2_xc(self.plan.h, self.prec, ptr(self.ao), ptr(self.weights), ptr(D), ptr(self.Vxc),
                          ptr(self.exc), stream_handle(stream)), "b2_xc")

    def fock_diis(self, use_diis=True, hyb=HYB_B3LYP, stream=None):
        check(lib().b2_fock_diis(self.plan.h, ptr(self.active), ptr(self.iter), float(hyb), int(use_diis),
                                 ptr(self.Hcore), ptr(self.S), ptr(self.D), ptr(self.J), ptr(self.K),
                                 ptr(self.Vxc), ptr(self.H), ptr(self.diffJK), ptr(self.ring_err),
                                 ptr(self.ring_h), ptr(self.bmat), ptr(self.diis_err),
                                 stream_handle(stream)), "b2_fock_diis")

    def eigh_density(self, stream=None):
        check(lib().b2_eigh_density(self.plan.h, ptr(self.active), ptr(self.H), ptr(self.Linv), ptr(self.D),
                                    ptr(self.mo_energy), ptr(self.C), ptr(self.sweeps),
                                    stream_handle(stream)), "b2_eigh_density")

    def energies(self, stream=None):
        check(lib().b2_energy(self.plan.h, ptr(self.active), ptr(self.D), ptr(self.Hcore), ptr(self.diffJK),
                              ptr(self.exc), ptr(self.enuc), ptr(self.energy), stream_handle(stream)),
              "b2_energy")

    def diff_jk(self, hyb=HYB_B3LYP):
        return self.J - 0.5 * hyb * self.K

    # --- SCF ----------------------------------------------------------------------------
    def prepare(self):
        if not self._eri_done:
            self.compute_eri()
        if not self._ao_done:
            self.compute_ao()

    def initial(self):
        """D <- D0, then XC and J/K of D0 (nanoDFT.py:146-148)."""
        self.D.copy_(self.D0)
        self.iter.zero_()
        self.active.fill_(1)
        self.xc()
        self.jk()

    def step(self, use_diis=True):
        """One SCF iteration for every active molecule (nanoDFT.py:63-80)."""
        self.fock_diis(use_diis)
        self.eigh_density()
        self.xc()
        self.jk()
        self.diffJK.copy_(self.diff_jk())
        self.energies()
        self.iter.add_(1)

    def run(self, its=20, use_diis=True, log=True):
        """Fixed-iteration SCF as in the reference (no convergence test, fori_loop of `its`)."""
        self.prepare()
        self.initial()
        P = self.plan
        nm = P.nmol
        E = torch.zeros((its, nm, 5), dtype=torch.float64, device=self.device)
        mo = torch.zeros((its, nm, NMO), dtype=torch.float64, device=self.device)
        derr = torch.zeros((its, nm), dtype=torch.float64, device=self.device)
        logs = []
        for i in range(its):
            self.step(use_diis)
            E[i] = self.energy.view(nm, 5)
            mo[i] = self.mo_energy.view(nm, NMO)
            derr[i] = self.diis_err
            if log:
                logs.append(torch.stack([self.D.clone(), self.diffJK.clone(), self.H.clone(), self.J.clone()]))
        out = dict(energies=E.cpu().numpy(), mo_energy=mo.cpu().numpy(), diis_err=derr.cpu().numpy())
        if log:
            out["logs"] = torch.stack(logs).cpu().numpy()      # (its, 4, n_mat): D, diff_JK, H, J
        out["C"] = self.C.cpu().numpy()
        return out

    def close(self):
        self.plan.close()
