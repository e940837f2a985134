"""Initial density matrix.

The reference starts SCF from PySCF's MINAO guess (``minao(mol)``, dft.py:223 ->
pyscf_utils/minao.py:5-123; ``init_guess_by_minao``, nanoDFT.py:233): the spherically
averaged ground-state occupations of each atom (``atom_hf.frac_occ``) placed in a
minimal ANO basis and projected onto the working basis.  For the minimal STO-3G basis
the projection keeps the same per-shell occupations on the atom's own AOs, so this
module places those occupations on the diagonal: H 1s^1; C/N/O/F 1s^2 2s^2 and the
2p electrons spread evenly over px, py, pz.
"""
import numpy as np

_P_ELECTRONS = {6: 2, 7: 3, 8: 4, 9: 5}


def minao_occupations(mol):
    occ = np.zeros(mol.nao)
    tab = mol.ao_table()
    for a in range(mol.nao):
        z = int(mol.charges[tab["atom"][a]])
        if z == 1:
            occ[a] = 1.0
        elif tab["l"][a] == 0:
            occ[a] = 2.0
        else:
            occ[a] = _P_ELECTRONS[z] / 3.0
    return occ


def minao(mol):
    """Drop-in for ``minao(mol)`` / ``init_guess_by_minao(mol)``: (nao, nao) float64."""
    return np.diag(minao_occupations(mol))
