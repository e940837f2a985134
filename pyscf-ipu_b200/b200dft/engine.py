"""Batched RKS engine on one B200: setup + device SCF loop through the C ABI.

One ``RKSEngine`` holds a batch of molecules (one molecule for the drop-in entry points).
Setup mirrors what the reference does on the host with PySCF before its jitted SCF
(dft.py:197-234, nanoDFT.py:208-257) -- molecule/basis (``Mole``), grid, one-electron
matrices, L = inv(cholesky(S)), MINAO-style guess, nuclear repulsion -- and runs on the
device by default (``setup="device"``) or on the host (``HostSetup`` list, numpy).  The SCF
loop runs entirely on the device: ERIs once, then per iteration Fock+DIIS, orthogonalised
eigensolve + density, XC and J/K, energies (nanoDFT.py:40-102).  ``run`` reproduces the
reference's fixed iteration count; ``run_converged`` iterates each molecule until its DIIS
error and energy change fall below thresholds and retires it (its kernels skip it).
"""
import ctypes
import numpy as np
import torch

from ._lib import lib, check, ptr, stream_handle, B200DFTError, launch_count, ScfState
from .constants import HYB_B3LYP
from .grids import Grids, atomic_grid
from .guess import minao
from .int1e import int1e

NMO = 72     # mo_energy row stride used by the device kernels
NZ = 10      # nuclear charges 0..9 indexed in the grid template table


_SIDE = {}


def _side_stream(device):
    """one high-priority side stream per device, shared by every engine: memory the caching
    allocator hands out on a stream is reused only by later allocations on that stream"""
    d = torch.device(device)
    key = d.index if d.index is not None else torch.cuda.current_device()
    if key not in _SIDE:
        _SIDE[key] = torch.cuda.Stream(torch.device("cuda", key), priority=-1)
    return _SIDE[key]


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
        args = (nmol, ptr(natm), ptr(nbas), ptr(atm), ptr(bas), ptr(env), ptr(env_off), ctypes.byref(h))
        rc = lib().b2_plan_create(*args)
        if rc == -2:
            # plan tables come from the driver's memory, which torch's caching allocator may be
            # holding after earlier batches: return torch's unused blocks and try once more
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            lib().b2_release_cached_memory()
            rc = lib().b2_plan_create(*args)
        check(rc, "b2_plan_create")
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
        self.epoch = 0                      # bumped by every launch-configuration change
        hb = ctypes.c_int64()
        check(lib().b2_plan_h2d_bytes(h, ctypes.byref(hb)), "b2_plan_h2d_bytes")
        self.h2d_bytes = hb.value

    def set_grid(self, npoints):
        goff = np.concatenate([[0], np.cumsum(npoints)]).astype(np.int64)
        rc = lib().b2_grid_set(self.h, ptr(goff))
        if rc == -2:                        # as in plan creation: torch's cache holds the memory
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            rc = lib().b2_grid_set(self.h, ptr(goff))
        check(rc, "b2_grid_set")
        self.epoch += 1
        npts, nao = ctypes.c_int64(), ctypes.c_int64()
        check(lib().b2_grid_info(self.h, ctypes.byref(npts), ctypes.byref(nao)), "b2_grid_info")
        self.grid_off = goff
        self.n_points, self.n_ao = npts.value, nao.value
        self.ao_off = np.zeros(self.nmol, np.int64)
        check(lib().b2_grid_ao_offsets(self.h, ptr(self.ao_off)), "b2_grid_ao_offsets")

    def set_jk_chunk(self, elems):
        check(lib().b2_plan_set_jk_chunk(self.h, int(elems)), "b2_plan_set_jk_chunk")
        self.epoch += 1

    def set_xc_impl(self, impl):
        """0 per-bucket persistent tensor-core kernel, 1 CUDA cores, 2 one-launch tensor cores"""
        check(lib().b2_plan_set_xc_impl(self.h, int(impl)), "b2_plan_set_xc_impl")
        self.epoch += 1

    def set_xc_tiles(self, tiles):
        check(lib().b2_plan_set_xc_tiles(self.h, int(tiles)), "b2_plan_set_xc_tiles")
        self.epoch += 1

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().b2_plan_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

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
    """Per-molecule host inputs (the reference's PySCF-side setup, numpy).  With
    ``ao_threshold`` > 0 the AO values are evaluated here, thresholded and the grid points left
    without any AO value are dropped (nanoDFT.py:221-230); ``ao`` then holds the (4, G, nao)
    values the SCF uses in place of on-the-fly ones."""

    def __init__(self, mol, level=0, grid=None, D0=None, ao_threshold=0.0):
        self.mol = mol
        S, T, V = int1e(mol)
        self.S, self.T, self.V = S, T, V
        self.Hcore = T + V
        self.L_inv = np.linalg.inv(np.linalg.cholesky(S))
        if grid is None:
            grid = Grids(mol, level).build()
        self.coords = np.ascontiguousarray(grid.coords, np.float64)
        self.weights = np.ascontiguousarray(grid.weights, np.float64)
        self.ao = None
        if ao_threshold and ao_threshold > 0.0:
            from .ao import eval_ao, threshold_grid
            self.ao, self.coords, self.weights = threshold_grid(eval_ao(mol, self.coords), self.coords,
                                                                self.weights, ao_threshold)
        self.D0 = minao(mol) if D0 is None else np.asarray(D0, np.float64)
        self.E_nuc = mol.energy_nuc()


_TEMPLATES = {}


def grid_templates(level):
    """Atom-centred grid templates (x, y, z, w) per nuclear charge for ``level``."""
    if level not in _TEMPLATES:
        parts, off = [], [0]
        for z in range(NZ):
            if z in (1, 6, 7, 8, 9):
                c, w = atomic_grid(z, level)
                parts.append(np.concatenate([c, w[:, None]], 1))
                off.append(off[-1] + len(w))
            else:
                off.append(off[-1])
        _TEMPLATES[level] = (np.ascontiguousarray(np.concatenate(parts)), np.array(off, np.int64))
    return _TEMPLATES[level]


class RKSEngine:
    """Device SCF for a batch of molecules.

    precision: "fp64" (plain: FP64 ERIs, J/K and grid path) or "mixed" (FP32 ERIs, J/K and
    grid path; FP64 Fock/DIIS/eigensolve/energies).
    setups: None (device setup) or a list of ``HostSetup``.
    """

    def __init__(self, mols, level=0, precision="fp64", setups=None, device=None, jk_chunk=None,
                 plan=None, guess="minao", net=None, eri_threshold=0.0, tuned=True):
        _require_cuda()
        self.mols = list(mols)
        self.level = level
        self.precision = precision
        self.prec = 64 if precision == "fp64" else 32
        self.device = torch.device(device or "cuda")
        self.setups = setups
        self.plan = plan if plan is not None else Plan(self.mols)
        if jk_chunk:
            self.plan.set_jk_chunk(jk_chunk)
        P = self.plan
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        rdt = torch.float64 if self.prec == 64 else torch.float32
        nm, nmat = P.nmol, P.n_mat
        z = lambda n: torch.zeros(n, **f64)
        if setups is not None:
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
            P.set_grid([len(s.weights) for s in setups])
            self.S = t(P.pack([s.S for s in setups]))
            self.Hcore = t(P.pack([s.Hcore for s in setups]))
            self.Linv = t(P.pack([s.L_inv for s in setups]))
            self.D0 = t(P.pack([s.D0 for s in setups]))
            self.coords = t(np.concatenate([s.coords for s in setups]).reshape(-1))
            self.weights = t(np.concatenate([s.weights for s in setups]))
            self.enuc = torch.tensor([s.E_nuc for s in setups], **f64)
            self._setup_done = True
        else:
            tmpl, toff = grid_templates(level)
            cnt = toff[1:] - toff[:-1]
            zall = np.concatenate([np.asarray(m.charges, np.int64) for m in self.mols])
            owner = np.repeat(np.arange(nm), [m.natm for m in self.mols])
            P.set_grid(np.bincount(owner, weights=cnt[zall], minlength=nm).astype(np.int64))
            self.S, self.T, self.V = z(nmat), z(nmat), z(nmat)
            self.Hcore, self.Linv, self.D0 = z(nmat), z(nmat), z(nmat)
            self.coords = z(3 * P.n_points)
            self.weights = z(max(1, P.n_points))
            self.enuc = z(nm)
            self.chol_status = torch.zeros(nm, dtype=torch.int32, device=dev)
            self._tmpl = (tmpl, toff)
            self._setup_done = False
        if tuned:                           # recorded autotuner choices of this device, if any
            from .autotune import apply
            apply(P)
        self.eri = torch.empty(max(1, P.n_eri), dtype=rdt, device=dev)
        self.eri_x = torch.empty(max(1, P.n_eri), dtype=rdt, device=dev)   # exchange list for J/K
        self.jk_impl = "pairs"      # "pairs": two products over the s8 and exchange lists; "s8"
        self.eri_threshold = float(eri_threshold or 0.0)   # > 0: |ERI| <= it become 0 (nanoDFT.py:280)
        self.ao = None          # (4, G, nao) AO tensor, only for the AO-input XC entry
        self.ao_stored = False  # the SCF's XC reads self.ao (thresholded host AO values)
        self._ao_done = False
        if setups is not None and any(getattr(s, "ao", None) is not None for s in setups):
            if not all(getattr(s, "ao", None) is not None for s in setups):
                raise ValueError("either every HostSetup of a batch carries AO values or none does")
            self.ao = torch.zeros(max(1, P.n_ao), dtype=rdt, device=dev)
            for m, s in enumerate(setups):
                o = int(P.ao_off[m])
                self.ao[o:o + s.ao.size] = torch.from_numpy(np.ascontiguousarray(s.ao).reshape(-1)).to(dev, rdt)
            self._ao_done = True
            self.ao_stored = True
        self.D, self.J, self.K, self.Vxc = z(nmat), z(nmat), z(nmat), z(nmat)
        self.H, self.diffJK = z(nmat), z(nmat)
        self.ring_err, self.ring_h = z(9 * nmat), z(9 * nmat)
        self.bmat = z(100 * nm)
        self.diis_err = z(nm)
        self.exc = z(nm)
        self.energy = z(5 * nm)
        self.mo_energy = z(NMO * nm)
        self.C = z(nmat)
        self.eig_ws = z(nmat)          # eigenvector basis carried between iterations (warm start)
        self.iter = torch.zeros(nm, dtype=torch.int32, device=dev)
        self.active = torch.ones(nm, dtype=torch.int32, device=dev)
        self.sweeps = torch.zeros(nm, dtype=torch.int32, device=dev)
        self._eri_done = False
        self._graph = None
        self.guess = guess                  # "minao" or "learned"
        self.net = net
        self.D0_minao = None
        self._guess_pending = False
        self._guess_after = self._guess_done = None
        self._side = None                   # side stream of the learned guess
        self.graph_replays = 0              # kernels replayed from graphs are not in launch_count()
        self._captured = 0
        self.graph_kernels_per_step = 0
        self._graph = None                  # (key, CUDAGraph) of one captured SCF iteration

    # --- setup -------------------------------------------------------------------------
    def device_setup(self, stream=None):
        """1e matrices, grid, guess, L and E_nuc on the device (no host round trip)."""
        if self._setup_done:
            return
        P, s = self.plan, stream_handle(stream)
        tmpl, toff = self._tmpl
        check(lib().b2_int1e(P.h, ptr(self.S), ptr(self.T), ptr(self.V), s), "b2_int1e")
        torch.add(self.T, self.V, out=self.Hcore)
        check(lib().b2_grid_build(P.h, NZ, ptr(tmpl), ptr(toff), ptr(self.coords), ptr(self.weights), s),
              "b2_grid_build")
        check(lib().b2_guess(P.h, ptr(self.D0), s), "b2_guess")
        check(lib().b2_enuc(P.h, ptr(self.enuc), s), "b2_enuc")
        check(lib().b2_chol_inv(P.h, ptr(self.S), ptr(self.Linv), ptr(self.chol_status), s), "b2_chol_inv")
        self._setup_done = True
        if self.guess == "learned":
            # the network runs after these kernels on a side stream, started by compute_eri
            # once the ERI kernels are queued (its host-side graph build then overlaps them)
            # or by initial(), whichever comes first
            cur = torch.cuda.current_stream(self.device)
            self._guess_after = cur.record_event()
            self._guess_pending = True

    def _start_guess(self):
        """queue a pending learned guess on a high-priority side stream after the setup kernels"""
        if not self._guess_pending:
            return
        self._guess_pending = False
        if self._side is None:
            self._side = _side_stream(self.device)
        self._side.wait_event(self._guess_after)
        if self.D0_minao is None:
            self.D0_minao = torch.empty_like(self.D0)
        with torch.cuda.stream(self._side):
            self.apply_learned_guess()
        self._guess_done = self._side.record_event()

    def apply_learned_guess(self):
        """D0 <- network prediction (MINAO kept as the fallback), on the current stream"""
        from .learned import Batch
        if self.net is None:
            from .train_guess import load
            self.net = load(device=self.device)
        if self.D0_minao is None:
            self.D0_minao = self.D0.clone()
        else:
            self.D0_minao.copy_(self.D0)
        if not hasattr(self, "_nn_batch"):
            self._nn_batch = Batch(self.mols, device=self.device, mat_off=self.plan.mat_off, nao=self.plan.nao)
        self.net.predict(self._nn_batch, self.D0)

    # --- kernels -----------------------------------------------------------------------
    def compute_eri(self, stream=None):
        check(lib().b2_eri_s8(self.plan.h, self.prec, ptr(self.eri), stream_handle(stream)), "b2_eri_s8")
        if self.eri_threshold > 0.0:
            check(lib().b2_eri_threshold(self.plan.h, self.prec, ptr(self.eri), self.eri_threshold,
                                         stream_handle(stream)), "b2_eri_threshold")
        check(lib().b2_jk_exchange(self.plan.h, self.prec, ptr(self.eri), ptr(self.eri_x), stream_handle(stream)),
              "b2_jk_exchange")
        self._eri_done = True
        self._start_guess()

    def compute_ao(self, stream=None):
        """Stored AO values + gradients (the reference's grid_AO tensor), for ``xc_from_ao``."""
        if self.ao is None:
            rdt = torch.float64 if self.prec == 64 else torch.float32
            self.ao = torch.empty(max(1, self.plan.n_ao), dtype=rdt, device=self.device)
        check(lib().b2_ao_eval(self.plan.h, self.prec, ptr(self.coords), ptr(self.ao),
                               stream_handle(stream)), "b2_ao_eval")
        self._ao_done = True

    def jk(self, D=None, active=None, stream=None):
        D = self.D if D is None else D
        if self.jk_impl == "s8":
            check(lib().b2_jk_s8(self.plan.h, self.prec, ptr(active), ptr(self.eri), ptr(D), ptr(self.J),
                                 ptr(self.K), stream_handle(stream)), "b2_jk_s8")
        else:
            check(lib().b2_jk_pairs(self.plan.h, self.prec, ptr(active), ptr(self.eri), ptr(self.eri_x), ptr(D),
                                    ptr(self.J), ptr(self.K), stream_handle(stream)), "b2_jk_pairs")

    def xc(self, D=None, active=None, stream=None):
        """E_xc and V_xc with AO values generated on the fly per grid tile."""
        D = self.D if D is None else D
        check(lib().b2_xc_direct(self.plan.h, self.prec, ptr(active), ptr(self.coords), ptr(self.weights),
                                 ptr(D), ptr(self.Vxc), ptr(self.exc), stream_handle(stream)), "b2_xc_direct")

    def scf_xc(self, active=None, stream=None):
        """the SCF's XC step: stored (thresholded) AO values when the setups carry them, else AO
        values generated per grid tile"""
        if self.ao_stored:
            self.xc_from_ao(active=active, stream=stream)
        else:
            self.xc(active=active, stream=stream)

    def xc_from_ao(self, D=None, active=None, stream=None):
        """E_xc and V_xc from the stored AO tensor (compute_ao first)."""
        D = self.D if D is None else D
        check(lib().b2_xc(self.plan.h, self.prec, ptr(active), ptr(self.ao), ptr(self.weights), ptr(D),
                          ptr(self.Vxc), ptr(self.exc), stream_handle(stream)), "b2_xc")

    def fock_diis(self, use_diis=True, hyb=HYB_B3LYP, stream=None):
        check(lib().b2_fock_diis(self.plan.h, ptr(self.active), ptr(self.iter), float(hyb), int(use_diis),
                                 ptr(self.Hcore), ptr(self.S), ptr(self.D), ptr(self.J), ptr(self.K),
                                 ptr(self.Vxc), ptr(self.H), ptr(self.diffJK), ptr(self.ring_err),
                                 ptr(self.ring_h), ptr(self.bmat), ptr(self.diis_err),
                                 stream_handle(stream)), "b2_fock_diis")

    def eigh_density(self, stream=None):
        check(lib().b2_eigh_density(self.plan.h, ptr(self.active), ptr(self.iter), ptr(self.H), ptr(self.Linv),
                                    ptr(self.D), ptr(self.mo_energy), ptr(self.C), ptr(self.eig_ws),
                                    ptr(self.sweeps), stream_handle(stream)), "b2_eigh_density")

    def energies(self, stream=None):
        check(lib().b2_energy(self.plan.h, ptr(self.active), ptr(self.D), ptr(self.Hcore), ptr(self.diffJK),
                              ptr(self.exc), ptr(self.enuc), ptr(self.energy), stream_handle(stream)),
              "b2_energy")

    # --- SCF ----------------------------------------------------------------------------
    def prepare(self):
        self.device_setup()
        if not self._eri_done:
            self.compute_eri()

    def initial(self):
        """D <- D0, then XC and J/K of D0 (nanoDFT.py:146-148)."""
        self._start_guess()
        if self._guess_done is not None:
            torch.cuda.current_stream(self.device).wait_event(self._guess_done)
            self._guess_done = None
        self.D.copy_(self.D0)
        self.iter.zero_()
        self.active.fill_(1)
        self.scf_xc()
        self.jk()

    def scf_state(self, use_diis=True, hyb=HYB_B3LYP):
        """the b2_scf_state of this engine's device buffers"""
        st = ScfState()
        for name, t in (("Hcore", self.Hcore), ("S", self.S), ("Linv", self.Linv), ("coords", self.coords),
                        ("weights", self.weights), ("enuc", self.enuc), ("eri", self.eri), ("D", self.D),
                        ("J", self.J), ("K", self.K), ("Vxc", self.Vxc), ("H", self.H), ("diffJK", self.diffJK),
                        ("ring_err", self.ring_err), ("ring_h", self.ring_h), ("bmat", self.bmat),
                        ("diis_err", self.diis_err), ("exc", self.exc), ("energy", self.energy),
                        ("mo_energy", self.mo_energy), ("C", self.C), ("eig_ws", self.eig_ws),
                        ("iter", self.iter), ("active", self.active), ("sweeps", self.sweeps)):
            setattr(st, name, t.data_ptr())
        st.ao = self.ao.data_ptr() if self.ao_stored else None
        st.exch = self.eri_x.data_ptr() if self.jk_impl == "pairs" else None
        st.hyb, st.use_diis, st.precision = float(hyb), int(use_diis), self.prec
        return st

    def _graph_key(self, use_diis):
        """what a captured iteration depends on: the buffers its launches read and write (fixed
        for the engine's life), the plan and its launch configuration"""
        st = self.scf_state(use_diis)
        return (self.plan.h.value, self.plan.epoch, self.ao_stored, self.jk_impl,
                tuple(getattr(st, f) for f, _ in ScfState._fields_))

    def drop_graph(self):
        """forget the captured iteration (after changing the plan's knobs through the C ABI)"""
        self._graph = None

    def step(self, use_diis=True):
        """One SCF iteration for every active molecule (nanoDFT.py:40-102): one b2_scf_iterate
        call (Fock + DIIS, eigensolve + density, XC, J/K, diff_JK, energies, iteration count)."""
        st = self.scf_state(use_diis)
        self._state = st                     # the call reads it synchronously; keep it referenced
        check(lib().b2_scf_iterate(self.plan.h, ctypes.byref(st), stream_handle()), "b2_scf_iterate")

    def step_entries(self, use_diis=True):
        """The same iteration as ``step`` through the individual entry points."""
        a = self.active
        self.fock_diis(use_diis)
        self.eigh_density()
        self.scf_xc(active=a)
        self.jk(active=a)
        torch.add(self.J, self.K, alpha=-0.5 * HYB_B3LYP, out=self.diffJK)
        self.energies()
        self.iter.add_(self.active)

    def run(self, its=20, use_diis=True, log=True):
        """Fixed-iteration SCF as in the reference (no convergence test, fori_loop of `its`)."""
        import time
        tm = {"initial": 0.0, "capture": 0.0, "graph_its": 0.0, "eager_its": 0.0, "restarts": 0}
        t = time.perf_counter()
        self.prepare()
        self.initial()
        tm["initial"] = 1e3 * (time.perf_counter() - t)
        nm = self.plan.nmol
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

    def run_converged(self, max_its=40, e_tol=1e-6, diis_tol=1e-4, use_diis=True, graph=True,
                      check_every=1, fallback=True, rise=3.0, fallback_window=5, tail=0.25,
                      after_capture=None):
        """Iterate until each molecule's |E_i - E_{i-1}| < e_tol and DIIS error < diis_tol, then
        retire it (its kernels skip it).  With a learned guess and ``fallback``, a molecule whose DIIS
        error rises by more than ``rise`` x from one iteration to the next during its first
        ``fallback_window`` iterations restarts once from MINAO.  Once at most ``tail`` of the batch
        is still iterating, the J/K and XC launches are compacted to those molecules (eager mode).
        Returns per-molecule energies, iterations (counted from the first start), flags and
        the energies of each molecule's last 5 iterations (``last5``, NaN where fewer ran).
        ``after_capture`` runs once the iteration graph is captured (or found in the cache; with
        ``graph=False`` once the initial evaluation is queued)."""
        import time
        tm = {"initial": 0.0, "capture": 0.0, "graph_its": 0.0, "eager_its": 0.0, "restarts": 0}
        t = time.perf_counter()
        self.prepare()
        self.initial()
        tm["initial"] = 1e3 * (time.perf_counter() - t)
        nm = self.plan.nmol
        dev = self.device
        e_prev = torch.full((nm,), float("inf"), dtype=torch.float64, device=dev)
        conv_it = torch.full((nm,), -1, dtype=torch.int32, device=dev)
        use_fb = fallback and self.D0_minao is not None
        sub_n = nm + 1
        fell_back = torch.zeros(nm, dtype=torch.bool, device=dev)
        err_prev = torch.full((nm,), float("inf"), dtype=torch.float64, device=dev)
        hist = torch.full((nm, 5), float("nan"), dtype=torch.float64, device=dev)   # last 5 energies
        g = None
        t = time.perf_counter()
        key = self._graph_key(use_diis) if graph else None
        if graph and self._graph is not None and self._graph[0] == key:
            g = self._graph[1]                       # same buffers and launch configuration
        elif graph:
            # capture one iteration (all launches go to the capture stream); replay per step
            self._graph = None
            st = torch.cuda.Stream()
            st.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            c0 = launch_count()
            with torch.cuda.stream(st):
                # explicit capture: torch.cuda.graph() would also run gc.collect() and release
                # the allocator cache (both slow for large batches, neither needed here).
                # Thread-local mode: another thread may build the next batch's plan (allocations,
                # copies, synchronisation) meanwhile without invalidating this capture.
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    self.step(use_diis)
                finally:
                    g.capture_end()
            torch.cuda.current_stream().wait_stream(st)
            self.graph_kernels_per_step = launch_count() - c0
            self._captured += self.graph_kernels_per_step
            self._graph = (key, g)
            # the capture did not execute the step: state is unchanged
        tm["capture"] = 1e3 * (time.perf_counter() - t)
        if after_capture is not None:
            after_capture()
        t = time.perf_counter()
        for i in range(max_its):
            if g is not None:
                g.replay()
                self.graph_replays += 1
            else:
                self.step(use_diis)
            e = self.energy.view(nm, 5)[:, 0]
            hist[:, i % 5] = torch.where(self.active > 0, e, hist[:, i % 5])
            newly = (self.active > 0) & ((e - e_prev).abs() < e_tol) & (self.diis_err < diis_tol)
            conv_it = torch.where(newly, torch.full_like(conv_it, i + 1), conv_it)
            self.active.masked_fill_(newly, 0)
            e_prev = torch.where(self.active > 0, e, e_prev)
            if use_fb:
                err = self.diis_err
                bad = ((self.active > 0) & ~fell_back & (self.iter >= 2) & (self.iter <= fallback_window)
                       & (err > rise * err_prev))
                err_prev = torch.where(self.active > 0, err, err_prev)
                if bool(bad.any()):
                    tm["restarts"] += 1
                    self._restart_from_minao(bad)
                    fell_back |= bad
                    e_prev = torch.where(bad, torch.full_like(e_prev, float("inf")), e_prev)
                    err_prev = torch.where(bad, torch.full_like(err_prev, float("inf")), err_prev)
            if (i + 1) % check_every == 0:
                n_act = int(self.active.sum().item())
                if n_act == 0:
                    break
                if n_act <= tail * nm and n_act <= sub_n // 2:
                    idx = self.active.nonzero().flatten().to(torch.int32).cpu().numpy()
                    check(lib().b2_plan_set_subset(self.plan.h, ptr(np.ascontiguousarray(idx)), len(idx)),
                          "b2_plan_set_subset")
                    sub_n = n_act
                    if g is not None:
                        tm["graph_its"] = 1e3 * (time.perf_counter() - t)
                        t = time.perf_counter()
                    g = None                                 # graph holds full-batch launches
        tm["graph_its" if g is not None else "eager_its"] = 1e3 * (time.perf_counter() - t)
        if sub_n <= nm:
            check(lib().b2_plan_set_subset(self.plan.h, None, 0), "b2_plan_set_subset")
        E = self.energy.view(nm, 5)[:, 0].clone()
        self.host_ms = tm                                # host wall time of the parts (ms)
        return dict(energy=E, iterations=conv_it, converged=conv_it > 0, mo_energy=self.mo_energy.view(nm, NMO),
                    diis_err=self.diis_err.clone(), its_run=i + 1, fell_back=fell_back, last5=hist)

    def _restart_from_minao(self, mask):
        """restart the molecules in ``mask`` from the MINAO density (iteration counter 0)"""
        P = self.plan
        sel = mask.nonzero().flatten().cpu().numpy()
        for m in sel:
            o, n = int(P.mat_off[m]), int(P.nao[m]) ** 2
            self.D[o:o + n].copy_(self.D0_minao[o:o + n])
        self.iter.masked_fill_(mask, 0)
        act = mask.to(torch.int32)
        self.scf_xc(active=act)
        self.jk(active=act)

    def gradient(self, parts=15, hyb=HYB_B3LYP, stream=None):
        """Nuclear gradients [Ha/Bohr] of the converged molecules from the final orbitals, on the
        engine's grid (``nuclear_gradient``): device float64 (sum of natm, 3)."""
        return nuclear_gradient(self.plan, self.C, self.mo_energy, self.coords, self.weights, parts=parts,
                                hyb=hyb, stream=stream)

    def kernels_launched(self, since):
        """library kernels executed since the launch_count() value ``since`` (graph replays included;
        the capture itself launches nothing)"""
        return launch_count() - since - self._captured + self.graph_replays * self.graph_kernels_per_step

    def close(self):
        self._graph = None
        self.plan.close()


def nuclear_gradient(plan, C, mo_energy, coords, weights, parts=15, hyb=HYB_B3LYP, stream=None, out_dm=None):
    """Nuclear gradients [Ha/Bohr] of converged SCFs, float64 on the device (b2_grad): the
    reference's grad = grad_elec + grad_nuc (nanoDFT.py:403-477) with the grid held fixed as
    there.  C (column k = orbital k) and mo_energy (``NMO`` per molecule) are laid out by
    ``plan``; coords / weights follow the grid registered with ``plan.set_grid``.  ``parts``
    selects terms (1 one-electron, 2 two-electron, 4 exchange-correlation, 8 nuclear
    repulsion).  Returns (sum of natm, 3), each molecule's atoms after those of the molecules
    before it; ``out_dm`` (a list) receives the dm0 and dme0 device matrices."""
    dev = C.device
    f64 = dict(dtype=torch.float64, device=dev)
    n_atm = sum(m.natm for m in plan.mols)
    D = torch.empty(max(1, plan.n_mat), **f64)
    W = torch.empty(max(1, plan.n_mat), **f64)
    g = torch.empty((max(1, n_atm), 3), **f64)
    check(lib().b2_grad(plan.h, int(parts), float(hyb), ptr(C), ptr(mo_energy), ptr(coords), ptr(weights),
                        ptr(D), ptr(W), ptr(g), stream_handle(stream)), "b2_grad")
    if out_dm is not None:
        out_dm.extend([D, W])
    return g[:n_atm]


def _run_one(mols, plan, level, precision, guess, net, run_kw, after_prepare=None, gradient=False):
    """one batch to convergence; returns host arrays, the engine's device memory released
    (back to the allocator cache, where the next batch's engine finds it).  ``after_prepare``
    runs once the batch's setup and ERI work is queued and its SCF iteration graph captured; with ``gradient`` the result also holds
    the nuclear gradients of the final orbitals (sum of natm x 3, Ha/Bohr)."""
    import time
    t0 = time.perf_counter()
    eng = RKSEngine(mols, level=level, precision=precision, guess=guess, net=net, plan=plan)
    try:
        t1 = time.perf_counter()
        eng.prepare()
        t2 = time.perf_counter()
        # the callback (the next batch's plan build on a worker thread) starts once this batch's
        # SCF iteration graph is captured: its CUDA calls then overlap the graph replays, not the
        # capture (a capture that waited on them left the GPU idle for up to 0.7 s)
        r = eng.run_converged(after_capture=after_prepare, **run_kw)
        out = {k: r[k].cpu().numpy() for k in ("energy", "iterations", "converged", "mo_energy",
                                               "last5", "diis_err")}
        t3 = time.perf_counter()
        if gradient:
            out["gradient"] = eng.gradient().cpu().numpy()
        out["its_run"] = r["its_run"]
        out["h2d_bytes"] = plan.h2d_bytes + getattr(getattr(eng, "_nn_batch", None), "h2d_bytes", 0)
        # host wall time of the batch's parts (ms): engine set-up, setup + ERI launch, SCF to results
        out["host_ms"] = {"engine": 1e3 * (t1 - t0), "prepare": 1e3 * (t2 - t1), "scf": 1e3 * (t3 - t2)}
        if gradient:
            out["host_ms"]["gradient"] = 1e3 * (time.perf_counter() - t3)
        out["host_ms"].update({"scf_" + k: v for k, v in getattr(eng, "host_ms", {}).items()})
        out["its_run"] = r["its_run"]
        return out
    finally:
        eng.close()


def run_batches(batches, level=0, precision="mixed", guess="learned", net=None, prefetch=True, gradient=False,
                **run_kw):
    """Run a sequence of molecule batches to convergence, one ``RKSEngine`` each, yielding
    ``(mols, result)`` per batch with the result's arrays on the host (energy, iterations,
    converged, mo_energy, last5, diis_err; with ``gradient`` also the nuclear gradients, the
    batch's atoms back to back).

    With ``prefetch`` the next batch's plan (host tables, upload and device table build on the
    plan's own stream) is made on a worker thread while the current batch runs on the GPU (from
    the moment its SCF iteration graph is captured); the C call releases the interpreter lock,
    so the two overlap.  ``run_kw`` goes to ``run_converged``; its ``graph`` defaults to False
    here: every batch has a new plan and new buffers, so a captured iteration graph would serve
    one batch only, and eager launches measured as fast on the B200 (11 417 vs 11 334
    molecules/s over 12 batches of 4096) without the capture's host time, which varied from 5
    to 700 ms between batches of one run."""
    run_kw.setdefault("graph", False)
    from concurrent.futures import ThreadPoolExecutor
    if guess == "learned" and net is None:
        from .train_guess import load
        net = load()
    it = iter(batches)
    dev = torch.cuda.current_device()

    def make(mols):
        torch.cuda.set_device(dev)          # worker threads start on device 0
        return list(mols), Plan(mols)

    ex = ThreadPoolExecutor(1) if prefetch else None
    try:
        import time
        tw = time.perf_counter()
        first = next(it, None)
        cur = None if first is None else make(first)
        wait_ms = 1e3 * (time.perf_counter() - tw)      # building the plan the next batch waited for
        while cur is not None:
            mols, plan = cur
            nxt = next(it, None)
            fut = []
            # the next plan's build starts once this batch's setup and ERI kernels are queued and
            # its iteration graph is captured, so it holds up neither
            start = (lambda: fut.append(ex.submit(make, nxt))) if (ex and nxt is not None) else None
            out = _run_one(mols, plan, level, precision, guess, net, run_kw, after_prepare=start,
                           gradient=gradient)
            out["host_ms"]["plan_wait"] = wait_ms
            del plan                      # the engine and plan are released before the next batch
            cur = None
            # the result goes out before the next plan is awaited: the caller's handling of it
            # overlaps the plan build, and a failing plan does not hold back a finished batch
            yield mols, out
            tw = time.perf_counter()
            if nxt is not None:
                cur = fut[0].result() if fut else make(nxt)
            wait_ms = 1e3 * (time.perf_counter() - tw)
    finally:
        if ex:
            ex.shutdown(wait=True)
