"""Initial density matrix: a diagonal approximation of the reference's MINAO guess.

The reference starts SCF from PySCF's MINAO guess (``minao(mol)``, dft.py:223 ->
pyscf_utils/minao.py:5-123; ``init_guess_by_minao``, nanoDFT.py:233): the spherically
averaged ground-state occupations of each atom (``atom_hf.frac_occ``) placed in a minimal ANO
basis and projected onto the working basis (``addons.project_dm_nr2nr(pmol, diag(occ), mol)``,
minao.py:116).  That projection goes through the overlap between the ANO and STO-3G functions,
so its result has off-diagonal and inter-atomic entries.  The ANO basis data and PySCF are not
available here, so this module keeps only the diagonal it approximates: the same per-shell
occupations on each atom's own AOs (H 1s^1; C/N/O/F 1s^2 2s^2 and the 2p electrons spread
evenly over px, py, pz).  It is an approximation of the reference's starting density, not the
same matrix; the SCF converges to the same solution from either, and the oracle, the device
kernel (b2_guess) and the tests all use this diagonal form.
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
