"""A numpy-backed stand-in for the few jax / PySCF / helper-package names the reference's
B3LYP, nanoDFT and sparse-s8 J/K modules use, so that those modules can be imported and run
UNMODIFIED in a container without jax 0.3.16 or pyscf 2.2.1 (fixture generation only; the
package never imports this).

jax parts (documented jax semantics, restated on numpy float64):
  * ``jax.jit`` / ``jax.pmap`` / ``jax.vmap``: function transforms.  ``jit`` is the identity;
    ``pmap`` runs one device (leading axis of size 1 stripped from the mapped inputs and put
    back on the outputs); ``vmap`` loops over the mapped axis.
  * ``jax.value_and_grad``: value and derivative of a scalar function, evaluated element-wise
    by the complex-step method (f'(x) = Im f(x + ih) / h, h = 1e-30 |x|; exact to rounding for
    the analytic functions b88/lyp/vwn/lda are built from).  The reference's vmap over points
    of ``value_and_grad`` of a scalar function is the same derivative per point.
  * ``jax.numpy.linalg.pinv``: singular values below 10 * max(M, N) * eps * s_max are dropped
    (jax's documented default rcond; numpy's default differs).
  * ``jax.lax``: ``fori_loop``, ``dynamic_update_slice``, ``psum`` (identity for one device),
    ``gather`` / ``scatter_add`` for one-dimensional operands with scalar index rows (the only
    form sparse_symmetric_ERI.py uses), ``bitcast_convert_type`` (numpy ``view``).
  * ``x.at[idx].set(v)`` / ``.mul(v)``: functional updates, provided by the ``AtArray``
    ndarray subclass that ``fori_loop`` gives to the arrays of its carried state.
Fakes of pyscf / chex / jaxtyping / jsonargparse / icecream / pyscf_ipu.nanoDFT.utils /
pyscf_ipu.electron_repulsion.direct provide only names that are imported, not called, plus a
``FakeMol`` / ``FakeGrids`` pair whose methods return this project's setup arrays (basis,
grid, one-electron integrals, MINAO-style guess) and the reference's own compiled ERIs.
"""
import dataclasses
import sys
import types

import numpy as np


# ------------------------------------------------------------------ functional array updates
class _At:
    def __init__(self, a):
        self.a = a

    def __getitem__(self, idx):
        return _AtIndex(self.a, idx)


class _AtIndex:
    def __init__(self, a, idx):
        self.a, self.idx = a, idx

    def set(self, v):
        out = np.array(self.a, copy=True).view(AtArray)
        out[self.idx] = v
        return out

    def mul(self, v):
        out = np.array(self.a, copy=True).view(AtArray)
        out[self.idx] = out[self.idx] * v
        return out

    def add(self, v):
        out = np.array(self.a, copy=True).view(AtArray)
        out[self.idx] = out[self.idx] + v
        return out


class AtArray(np.ndarray):
    @property
    def at(self):
        return _At(self)


def _at(x):
    """carry arrays inside lists / tuples / dicts as AtArray (jax arrays have ``.at``)"""
    if isinstance(x, np.ndarray) and not isinstance(x, AtArray):
        return x.view(AtArray)
    if isinstance(x, list):
        return [_at(v) for v in x]
    if isinstance(x, tuple):
        return tuple(_at(v) for v in x)
    if isinstance(x, dict):
        return {k: _at(v) for k, v in x.items()}
    return x


# ------------------------------------------------------------------ jax.numpy
def _make_jnp():
    jnp = types.ModuleType("jax.numpy")
    for name in dir(np):
        if not name.startswith("_"):
            setattr(jnp, name, getattr(np, name))
    lin = types.ModuleType("jax.numpy.linalg")
    for name in dir(np.linalg):
        if not name.startswith("_"):
            setattr(lin, name, getattr(np.linalg, name))

    def pinv(a, rcond=None):
        a = np.asarray(a)
        if rcond is None:
            rcond = 10 * max(a.shape[-2:]) * np.finfo(a.dtype).eps
        return np.linalg.pinv(a, rcond=rcond)

    lin.pinv = pinv
    jnp.linalg = lin

    def array(x, dtype=None):
        return np.array(x, dtype=dtype).view(AtArray)

    jnp.array = array
    jnp.zeros = lambda *a, **k: np.zeros(*a, **k).view(AtArray)
    jnp.ones = lambda *a, **k: np.ones(*a, **k).view(AtArray)
    return jnp


# ------------------------------------------------------------------ jax transforms
def _complex_step(f, args, wrt):
    h = 1e-30
    a = [np.asarray(x, dtype=np.complex128) for x in args]
    scale = np.maximum(np.abs(np.asarray(args[wrt], np.float64)), 1e-300)
    a[wrt] = a[wrt] + 1j * h * scale
    v = f(*a)
    return np.real(v), np.imag(v) / (h * scale)


def value_and_grad(f, argnums=0):
    def g(*args):
        nums = argnums if isinstance(argnums, tuple) else (argnums,)
        val = None
        grads = []
        for k in nums:
            v, d = _complex_step(f, args, k)
            val = v if val is None else val
            grads.append(d)
        return val, (tuple(grads) if isinstance(argnums, tuple) else grads[0])
    g._elementwise = True           # the reference differentiates element-wise scalar functions
    return g


def vmap(f, in_axes=0):
    def g(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.asarray(a).shape[ax]
                break
        # element-wise scalar functions (b3lyp's lda/vwn/b88/lyp): one call on whole arrays
        if all(ax in (0, None) for ax in axes) and getattr(f, "_elementwise", False):
            return f(*args)
        outs = []
        for t in range(n):
            outs.append(f(*[np.take(np.asarray(a), t, axis=ax) if ax is not None else a
                            for a, ax in zip(args, axes)]))
        if isinstance(outs[0], tuple):
            return tuple(_stack([o[k] for o in outs]) for k in range(len(outs[0])))
        return _stack(outs)
    return g


def _stack(xs):
    if isinstance(xs[0], tuple):
        return tuple(_stack([x[k] for x in xs]) for k in range(len(xs[0])))
    return np.stack([np.asarray(x) for x in xs]).view(AtArray)


def jit(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def pmap(f, in_axes=0, axis_name=None, **kw):
    def g(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)

        def strip(a, ax):
            if ax is None:
                return a
            if isinstance(ax, (list, tuple)):
                return [strip(x, y) for x, y in zip(a, ax)]
            return np.asarray(a)[0]
        out = f(*[strip(a, ax) for a, ax in zip(args, axes)])
        return [np.asarray(o)[None] for o in out]
    return g


def _make_lax():
    lax = types.ModuleType("jax.lax")

    def fori_loop(lo, hi, body, init):
        val = _at(init)
        for i in range(lo, hi):
            val = _at(body(i, val))
        return val

    def dynamic_update_slice(a, upd, idx):
        out = np.array(a, copy=True).view(AtArray)
        sl = tuple(slice(int(s), int(s) + n) for s, n in zip(idx, np.shape(upd)))
        out[sl] = upd
        return out

    class _Dn:
        def __init__(self, **k):
            self.__dict__.update(k)

    class GatherScatterMode:
        FILL_OR_DROP = "fill_or_drop"

    def gather(operand, idx, dimension_numbers=None, slice_sizes=None, mode=None, **kw):
        operand = np.asarray(operand)
        i = np.asarray(idx).reshape(-1).astype(np.int64)
        ok = (i >= 0) & (i < operand.shape[0])
        out = np.zeros(i.shape, operand.dtype)
        out[ok] = operand[i[ok]]
        return out.view(AtArray)

    def scatter_add(operand, idx, updates, dimension_numbers=None, mode=None, **kw):
        out = np.array(operand, copy=True)
        i = np.asarray(idx).reshape(-1).astype(np.int64)
        u = np.asarray(updates).reshape(-1)
        ok = (i >= 0) & (i < out.shape[0])
        np.add.at(out, i[ok], u[ok])
        return out.view(AtArray)

    lax.fori_loop = fori_loop
    lax.dynamic_update_slice = dynamic_update_slice
    lax.psum = lambda x, axis_name=None: x
    lax.GatherDimensionNumbers = _Dn
    lax.ScatterDimensionNumbers = _Dn
    lax.GatherScatterMode = GatherScatterMode
    lax.gather = gather
    lax.scatter_add = scatter_add
    lax.bitcast_convert_type = lambda x, dt: np.asarray(x).view(dt)
    return lax


def install():
    """put the stand-in modules into sys.modules (before importing reference modules)"""
    jax = types.ModuleType("jax")
    jax.numpy = _make_jnp()
    jax.lax = _make_lax()
    jax.jit = jit
    jax.pmap = pmap
    jax.vmap = vmap
    jax.value_and_grad = value_and_grad
    jax.checkpoint = lambda f: f
    jax.debug = types.SimpleNamespace(callback=lambda *a, **k: None)
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None, FLAGS=types.SimpleNamespace())
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jax.numpy
    sys.modules["jax.lax"] = jax.lax

    # imported-only names of packages absent here
    pyscf = types.ModuleType("pyscf")
    pyscf.dft = types.SimpleNamespace(gen_grid=types.SimpleNamespace(Grids=FakeGrids))
    pyscf.scf = types.SimpleNamespace(hf=types.SimpleNamespace(init_guess_by_minao=lambda mol: mol.minao()))
    sys.modules["pyscf"] = pyscf
    chex = types.ModuleType("chex")
    chex.dataclass = dataclasses.dataclass
    sys.modules["chex"] = chex
    jt = types.ModuleType("jaxtyping")

    class _Sub:
        def __getitem__(self, k):
            return object
    jt.Float = jt.Int = _Sub()
    jt.Array = object
    sys.modules["jaxtyping"] = jt
    ja = types.ModuleType("jsonargparse")
    ja.CLI = lambda *a, **k: None
    ja.Namespace = types.SimpleNamespace
    sys.modules["jsonargparse"] = ja
    ic = types.ModuleType("icecream")
    ic.ic = lambda *a, **k: a
    sys.modules["icecream"] = ic
    utils = types.ModuleType("pyscf_ipu.nanoDFT.utils")
    sys.modules["pyscf_ipu.nanoDFT.utils"] = utils
    direct = types.ModuleType("pyscf_ipu.electron_repulsion.direct")
    direct.prepare_electron_repulsion_integrals = direct.electron_repulsion_integrals = None
    direct.ipu_einsum = None
    sys.modules["pyscf_ipu.electron_repulsion.direct"] = direct
    return jax


# ------------------------------------------------------------------ PySCF-shaped inputs
class FakeGrids:
    """``pyscf.dft.gen_grid.Grids(mol)`` returning the molecule's precomputed grid"""

    def __init__(self, mol):
        self.mol = mol
        self.level = 0

    def build(self):
        self.coords, self.weights = self.mol.grid(self.level)
        return self


class FakeMol:
    """The PySCF ``Mole`` methods nanoDFT's setup calls (nanoDFT.py:208-257, 283-285), answered
    with this project's setup arrays and the reference's compiled ERIs (s8 / dense)."""

    cart = False

    def __init__(self, mole, grid_fn, ao_fn, int1e_fn, minao_fn, eri_s8_fn, unpack_fn):
        self.m = mole
        self._grid, self._ao, self._int1e, self._minao = grid_fn, ao_fn, int1e_fn, minao_fn
        self._eri_s8, self._unpack = eri_s8_fn, unpack_fn
        self.nelectron = mole.nelectron
        self._cache = {}

    def nao_nr(self):
        return self.m.nao

    def energy_nuc(self):
        return self.m.energy_nuc()

    def grid(self, level):
        return self._grid(self.m, level)

    def eval_gto(self, name, coords, comp):
        assert name == "GTOval_sph_deriv1" and comp == 4
        return self._ao(self.m, coords)

    def intor_symmetric(self, name):
        S, T, V = self._int1e(self.m)
        return {"int1e_ovlp": S, "int1e_kin": T, "int1e_nuc": V}[name]

    def minao(self):
        return self._minao(self.m)

    def intor(self, name, aosym="s1"):
        assert name == "int2e_sph"
        if "s8" not in self._cache:
            self._cache["s8"] = self._eri_s8(self.m)
        s8 = self._cache["s8"].copy()
        return s8 if aosym == "s8" else self._unpack(s8, self.m.nao)
