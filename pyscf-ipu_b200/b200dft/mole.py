"""A minimal ``Mole``: atoms, STO-3G shells and the libcint atm/bas/env arrays.

This replaces the PySCF ``Mole`` that the reference builds on the host
(pyscf_utils/build_mol.py:5-129, dft.py:1307, nanoDFT.py:543-546) with just what the
RKS hot path reads from it: ``nao_nr``, ``nelectron``, ``energy_nuc``, the atom
charges and coordinates (Bohr) and the libcint arrays that the reference packs
for its ERI kernels (``prepare_int_floats``, electron_repulsion/direct.py:710-739).
"""
import re
import numpy as np

from .constants import (ANGSTROM_TO_BOHR, ATM_SLOTS, BAS_SLOTS, CHARGE_OF, PTR_COORD,
                        ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, PTR_EXP, PTR_COEFF,
                        PTR_ENV_START, ELEMENTS, SYMBOLS)
from .basis import get_basis, normalized_coefficients


def parse_atom_string(atom):
    """Parse "C 0 0 0; H 0 0 1.09" (or a list of (symbol, xyz)) into symbols, coords."""
    if isinstance(atom, str):
        items = []
        for part in re.split(r"[;\n]", atom):
            toks = part.replace(",", " ").split()
            if not toks:
                continue
            if len(toks) != 4:
                raise ValueError(f"cannot parse atom entry '{part}'")
            items.append((toks[0], tuple(float(t) for t in toks[1:])))
    else:
        items = [(a[0], tuple(float(x) for x in a[1])) for a in atom]
    syms, xyz = [], []
    for s, c in items:
        s = s.strip()
        s = s[0].upper() + s[1:].lower()
        if s not in ELEMENTS:
            raise ValueError(f"element '{s}' is not supported")
        syms.append(s)
        xyz.append(c)
    return syms, np.asarray(xyz, dtype=np.float64).reshape(-1, 3)


class Mole:
    """Restricted closed-shell molecule in a contracted Gaussian basis.

    Attributes mirror the PySCF fields the reference reads: ``_atm``, ``_bas``,
    ``_env`` (int32 / float64, libcint slot layout), ``ao_loc``.
    """

    def __init__(self, atom, basis="sto-3g", unit="Angstrom", charge=0, spin=0):
        if spin != 0:
            raise ValueError("only closed-shell (spin=0) molecules are supported")
        self.basis = basis
        self.unit = unit
        self.charge = int(charge)
        self.spin = 0
        self.symbols, xyz = parse_atom_string(atom)
        scale = ANGSTROM_TO_BOHR if unit.lower().startswith("a") else 1.0
        self.coords = xyz * scale                      # Bohr
        self.charges = np.array([ELEMENTS[s] for s in self.symbols], dtype=np.int32)
        self.natm = len(self.symbols)
        self._build_env()
        if self.nelectron % 2:
            raise ValueError("odd electron count: restricted closed shell needs an even count")

    # --- libcint arrays -------------------------------------------------------------
    def _build_env(self):
        bset = get_basis(self.basis)
        env = [0.0] * PTR_ENV_START
        atm = np.zeros((self.natm, ATM_SLOTS), dtype=np.int32)
        for ia in range(self.natm):
            atm[ia, CHARGE_OF] = self.charges[ia]
            atm[ia, PTR_COORD] = len(env)
            env.extend(self.coords[ia].tolist())
            atm[ia, 2] = 1                             # point nucleus
            atm[ia, 3] = len(env)
            env.append(0.0)                            # nuclear zeta (unused)
        elem_ptr = {}
        bas = []
        for ia, s in enumerate(self.symbols):
            if s not in elem_ptr:
                ptrs = []
                for l, exps, coefs in bset[s]:
                    pe = len(env)
                    env.extend(exps)
                    pc = len(env)
                    env.extend(normalized_coefficients(l, exps, coefs).tolist())
                    ptrs.append((l, len(exps), pe, pc))
                elem_ptr[s] = ptrs
            for l, nprim, pe, pc in elem_ptr[s]:
                row = np.zeros(BAS_SLOTS, dtype=np.int32)
                row[ATOM_OF], row[ANG_OF], row[NPRIM_OF], row[NCTR_OF] = ia, l, nprim, 1
                row[PTR_EXP], row[PTR_COEFF] = pe, pc
                bas.append(row)
        self._atm = atm
        self._bas = np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS)
        self._env = np.asarray(env, dtype=np.float64)
        self.nbas = self._bas.shape[0]
        dims = 2 * self._bas[:, ANG_OF] + 1
        self.ao_loc = np.concatenate([[0], np.cumsum(dims)]).astype(np.int32)

    # --- PySCF-like accessors ---------------------------------------------------------
    def nao_nr(self):
        return int(self.ao_loc[-1])

    @property
    def nao(self):
        return self.nao_nr()

    @property
    def nelectron(self):
        return int(self.charges.sum()) - self.charge

    def atom_charges(self):
        return self.charges.copy()

    def atom_coords(self):
        return self.coords.copy()

    def atom_symbol(self, ia):
        return self.symbols[ia]

    def energy_nuc(self):
        """Nuclear repulsion sum_{a<b} Z_a Z_b / r_ab (experimental/structure.py:81-99)."""
        z = self.charges.astype(np.float64)
        d = self.coords[:, None, :] - self.coords[None, :, :]
        r = np.sqrt((d * d).sum(-1))
        iu = np.triu_indices(self.natm, 1)
        return float((z[iu[0]] * z[iu[1]] / r[iu]).sum())

    def aoslice_by_atom(self):
        out = np.zeros((self.natm, 4), dtype=np.int64)
        for ia in range(self.natm):
            sh = np.where(self._bas[:, ATOM_OF] == ia)[0]
            out[ia] = (sh[0], sh[-1] + 1, self.ao_loc[sh[0]], self.ao_loc[sh[-1] + 1])
        return out

    # --- per-AO tables used by the device kernels --------------------------------------
    def ao_table(self):
        """Per-AO description: (atom, l, component, nprim, exps[3], coefs[3]).

        ``component`` is 0 for s and 0/1/2 for px/py/pz.  Coefficients are the
        libcint ones multiplied by the angular factor, so that
        AO(r) = sum_i c_i * (x-X)^{cx} (y-Y)^{cy} (z-Z)^{cz} * exp(-a_i |r-R|^2).
        """
        from .constants import COMMON_FAC_SP
        n = self.nao
        atom = np.zeros(n, np.int32)
        lval = np.zeros(n, np.int32)
        comp = np.zeros(n, np.int32)
        exps = np.zeros((n, 3), np.float64)
        coef = np.zeros((n, 3), np.float64)
        for ish in range(self.nbas):
            ia, l, npr = self._bas[ish, ATOM_OF], self._bas[ish, ANG_OF], self._bas[ish, NPRIM_OF]
            pe, pc = self._bas[ish, PTR_EXP], self._bas[ish, PTR_COEFF]
            for c in range(2 * l + 1):
                a = self.ao_loc[ish] + c
                atom[a], lval[a], comp[a] = ia, l, c
                exps[a, :npr] = self._env[pe:pe + npr]
                coef[a, :npr] = self._env[pc:pc + npr] * COMMON_FAC_SP[l]
        return dict(atom=atom, l=lval, comp=comp, exps=exps, coef=coef)

    def __repr__(self):
        return f"Mole(natm={self.natm}, nao={self.nao}, nelectron={self.nelectron})"


def pack_moles(mols):
    """The molecules' arrays concatenated into a few flat arrays: the form in which generation
    workers send a chunk of molecules (one pickle of a few arrays instead of several small
    arrays per molecule; unpickling Mole objects cost 65 us each)."""
    cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs), dtype=dt) if xs else np.zeros(0, dt)
    return {
        "natm": np.array([m.natm for m in mols], np.int32),
        "nbas": np.array([m.nbas for m in mols], np.int32),
        "nenv": np.array([len(m._env) for m in mols], np.int64),
        "charge": np.array([m.charge for m in mols], np.int32),
        "basis": [m.basis for m in mols], "unit": [m.unit for m in mols],
        "coords": cat([m.coords for m in mols], np.float64).reshape(-1, 3),
        "charges": cat([m.charges for m in mols], np.int32),
        "atm": cat([m._atm for m in mols], np.int32).reshape(-1, ATM_SLOTS),
        "bas": cat([m._bas for m in mols], np.int32).reshape(-1, BAS_SLOTS),
        "env": cat([m._env for m in mols], np.float64),
        "ao_loc": cat([m.ao_loc for m in mols], np.int32),
    }


def unpack_moles(p):
    """Mole objects whose arrays are views into the packed arrays (no parsing, no basis build)."""
    out = []
    a0 = b0 = e0 = 0
    for k in range(len(p["natm"])):
        na, nb, ne = int(p["natm"][k]), int(p["nbas"][k]), int(p["nenv"][k])
        m = Mole.__new__(Mole)
        m.basis, m.unit, m.charge, m.spin = p["basis"][k], p["unit"][k], int(p["charge"][k]), 0
        m.coords = p["coords"][a0:a0 + na]
        m.charges = p["charges"][a0:a0 + na]
        m.symbols = [SYMBOLS[int(z)] for z in m.charges]
        m.natm, m.nbas = na, nb
        m._atm = p["atm"][a0:a0 + na]
        m._bas = p["bas"][b0:b0 + nb]
        m._env = p["env"][e0:e0 + ne]
        m.ao_loc = p["ao_loc"][b0 + k:b0 + k + nb + 1]
        out.append(m)
        a0, b0, e0 = a0 + na, b0 + nb, e0 + ne
    return out


def build_mol(mol_str, basis_name="sto-3g", unit="Angstrom"):
    """Drop-in for ``build_mol`` (nanoDFT.py:543-546)."""
    return Mole(mol_str, basis=basis_name, unit=unit)


def methane(ch=1.09):
    """CH4: C at the origin, 4 H along (+-1,+-1,+-1)/sqrt(3) at ``ch`` Angstrom."""
    d = ch / np.sqrt(3.0)
    pos = [(0, 0, 0), (d, d, d), (-d, -d, d), (-d, d, -d), (d, -d, -d)]
    return "C %f %f %f; " % pos[0] + "; ".join("H %.10f %.10f %.10f" % p for p in pos[1:])
