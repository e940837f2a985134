"""CLI shim: ``python density_functional_theory.py -methane`` / ``-str '...'`` runs the B200
RKS driver (b200dft.dft), mirroring ``pyscf_ipu/dft.py``'s command line."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "pyscf-ipu_b200"))

from b200dft.dft import main, density_functional_theory, jax_dft, get_args  # noqa: E402,F401

if __name__ == "__main__":
    main()
