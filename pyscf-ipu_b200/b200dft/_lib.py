"""ctypes binding of libb200dft.so (the C ABI declared in include/b200dft.h).

The product path has no CPU fallback: if the library is missing or no CUDA device is
present, calls raise ``B200DFTError``.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libb200dft.so")
HOSTCHECK_PATH = os.path.join(_HERE, "_lib", "libb200dft_hostcheck.so")

ERRORS = {-1: "bad argument", -2: "CUDA error", -3: "unsupported basis/shell", -4: "size limit exceeded",
          -5: "overlap matrix not positive definite", -6: "device wait timed out"}

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_D = ctypes.c_double

# name -> argtypes (all return int status)
SIGNATURES = {
    "b2_version": [],
    "b2_release_cached_memory": [],
    "b2_launch_count": [_P],
    "b2_plan_create": [_I, _P, _P, _P, _P, _P, _P, _P],
    "b2_plan_destroy": [_P],
    "b2_plan_info": [_P, _P],
    "b2_plan_h2d_bytes": [_P, _P],
    "b2_plan_offsets": [_P, _P, _P, _P, _P],
    "b2_plan_set_jk_chunk": [_P, _L],
    "b2_plan_set_xc_impl": [_P, _I],
    "b2_plan_set_xc_tiles": [_P, _I],
    "b2_plan_set_xc_bucket_tiles": [_P, _P],
    "b2_xc_tc_status": [_I, _P],
    "b2_nn_gemm_status": [_I, _P],
    "b2_jk_status": [_I, _P],
    "b2_plan_set_subset": [_P, _P, _I],
    "b2_eri_s8": [_P, _I, _P, _P],
    "b2_jk_s8": [_P, _I, _P, _P, _P, _P, _P, _P],
    "b2_jk_exchange": [_P, _I, _P, _P, _P],
    "b2_jk_pairs": [_P, _I, _P, _P, _P, _P, _P, _P, _P],
    "b2_grid_set": [_P, _P],
    "b2_grid_info": [_P, _P, _P],
    "b2_grid_ao_offsets": [_P, _P],
    "b2_ao_eval": [_P, _I, _P, _P, _P],
    "b2_xc": [_P, _I, _P, _P, _P, _P, _P, _P, _P],
    "b2_xc_direct": [_P, _I, _P, _P, _P, _P, _P, _P, _P],
    "b2_b3lyp": [_L, _P, _P, _P, _P, _P],
    "b2_chol_inv": [_P, _P, _P, _P, _P],
    "b2_fock_diis": [_P, _P, _P, _D, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "b2_eigh_density": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "b2_energy": [_P, _P, _P, _P, _P, _P, _P, _P, _P],
    "b2_int2e_sph_s8": [_P, _I, _P, _I, _P, _I, _I, _P, _P],
    "b2_int2e_sph_s8_noalloc": [_P, _I, _P, _I, _P, _I, _I, _P, _P],
    "b2_int1e": [_P, _P, _P, _P, _P],
    "b2_grid_build": [_P, _I, _P, _P, _P, _P, _P],
    "b2_guess": [_P, _P, _P],
    "b2_enuc": [_P, _P, _P],
    "b2_grad": [_P, _I, _D, _P, _P, _P, _P, _P, _P, _P, _P],
    "b2_eri_threshold": [_P, _I, _P, _D, _P],
    "b2_scf_iterate": [_P, _P, _P],
    "b2_copy_blocks": [_I, _P, _P, _P, _P, _P, _P],
    "b2_eri_work": [_P, _P],
    "b2_fp32_peak": [_P],
}


class ScfState(ctypes.Structure):
    """b2_scf_state (include/b200dft.h): device pointers of a batch's SCF state"""
    _fields_ = ([(n, _P) for n in ("Hcore", "S", "Linv", "coords", "weights", "enuc", "ao", "eri", "exch",
                                   "D", "J", "K", "Vxc", "H", "diffJK", "ring_err", "ring_h", "bmat",
                                   "diis_err", "exc", "energy", "mo_energy", "C", "eig_ws",
                                   "iter", "active", "sweeps")] +
                [("hyb", _D), ("use_diis", _I), ("precision", _I)])


class B200DFTError(RuntimeError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise B200DFTError(f"{LIB_PATH} not found: build it with `python pyscf-ipu_b200/csrc/build.py` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.b2_last_error.restype = ctypes.c_char_p
        L.b2_last_error.argtypes = []
        _lib = L
    return _lib


def check(rc, what):
    if rc != 0:
        detail = ""
        try:
            detail = lib().b2_last_error().decode()
        except Exception:
            pass
        raise B200DFTError(f"{what} failed: {ERRORS.get(rc, rc)} {detail}".strip())
    return rc


def launch_count():
    """kernels launched by libb200dft.so so far in this process"""
    v = ctypes.c_int64()
    check(lib().b2_launch_count(ctypes.byref(v)), "b2_launch_count")
    return v.value


def ptr(t):
    """device/host pointer of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return ctypes.c_void_p(t.ctypes.data)


def stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
