"""ctypes bindings of lib/libqcgpu.so and lib/libqsym.so (fail loudly if absent)."""
import ctypes
import os

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

c_int = ctypes.c_int
c_ll = ctypes.c_longlong
c_vp = ctypes.c_void_p
c_dbl = ctypes.c_double
c_char_p = ctypes.c_char_p

TASK_BYTES = 64
CONTRIB_BYTES = 80
OP_BYTES = 32
GROUP_BGEMM, GROUP_PANEL, GROUP_FIBER = 1, 2, 3     # work-item group kinds (qc_types.h)


class NativeError(RuntimeError):
    pass


def _load(name):
    path = os.path.join(LIBDIR, name)
    if not os.path.exists(path):
        raise NativeError("%s is missing: build it with `python -m qcmpodmrg_b200.build` "
                          "(there is no CPU fallback)" % path)
    return ctypes.CDLL(path)


_lib = None
_qsym = None

_SIGS = {
    "qc_version": (c_int, []),
    "qc_last_error": (c_char_p, []),
    "qc_last_cuda_error": (c_char_p, []),
    "qc_sym_allowed": (c_int, [c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "qc_sym_allowed_gpu": (c_int, [c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "qc_block_layout": (c_int, [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "qc_psi_diag_gather": (c_int, [c_ll, c_vp, c_vp, c_vp, c_vp, c_ll, c_ll, c_ll, c_vp]),
    "qc_contract_pairs": (c_ll, [c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_ll]),
    "qc_compile_pairs": (c_ll, [c_int, c_vp, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp, c_vp, c_vp,
                                c_int, c_vp, c_vp, c_ll, c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_int,
                                c_int, c_int, c_vp, c_ll, c_vp, c_ll, c_vp, c_vp]),
    "qc_bgemm_f64": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_bgemm_f32": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_bgemm_tf32": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_bgemm_tf32x3": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_gather_f64": (c_int, [c_vp, c_vp, c_vp, c_ll, c_vp]),
    "qc_reduce_ops_f64": (c_int, [c_vp, c_int, c_ll, c_vp, c_vp]),
    "qc_tc_status": (c_int, []),
    "qc_pgemm_f64": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_pgemm_f32": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_block_permute": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_int, c_vp]),
    "qc_fiber_f64": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "qc_fiber_f32": (c_int, [c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "qc_mlp_forward": (c_int, [c_int, c_int] + [c_vp] * 10 + [c_vp]),
    "qc_mlp_backward": (c_int, [c_int, c_int] + [c_vp] * 12 + [c_vp]),
    "qc_adam_step": (c_int, [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                             ctypes.c_float, c_int, ctypes.c_float, c_vp]),
    "qc_precond_apply": (c_int, [c_ll, c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp, c_vp]),
    "qc_sigma_f64_noalloc": (c_int, [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                     c_vp, c_vp, c_vp, c_int, c_ll, c_ll, c_ll, c_ll, c_vp]),
    "qc_reduce_ops_f32": (c_int, [c_vp, c_int, c_ll, c_vp, c_vp]),
    "qc_scatter_f64": (c_int, [c_vp, c_vp, c_vp, c_ll, c_ll, c_vp]),
    "qc_convert_f64_to_f32": (c_int, [c_vp, c_vp, c_ll, c_vp]),
    "qc_convert_f32_to_f64": (c_int, [c_vp, c_vp, c_ll, c_vp]),
    "qc_tmap_encode": (c_int, [c_int, c_vp, c_vp]),
    "qc_tcpanel_f32": (c_int, [c_vp, c_ll, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "qc_tf32_split": (c_int, [c_vp, c_vp, c_ll, c_vp]),
    "qc_tcpanel_status": (c_int, [c_int]),
    "qc_tcpanel_seg_f32": (c_int, [c_vp, c_ll, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "qc_gather_split_f32": (c_int, [c_vp, c_vp, c_ll, c_vp, c_vp, c_vp]),
    "qc_fgemm_f64": (c_int, [c_vp, c_ll, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "qc_fgemm_f32": (c_int, [c_vp, c_ll, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "qc_wpanel_f64": (c_int, [c_vp, c_vp, c_vp, c_ll, c_vp]),
    "qc_wpanel_f32": (c_int, [c_vp, c_vp, c_vp, c_ll, c_vp]),
    "qc_wpanel_pairs_f64": (c_int, [c_vp, c_ll, c_vp, c_ll, c_int, c_vp, c_vp, c_ll, c_vp]),
    "qc_wpanel_pairs_f32": (c_int, [c_vp, c_ll, c_vp, c_ll, c_int, c_vp, c_vp, c_ll, c_vp]),
}


def lib():
    global _lib
    if _lib is None:
        l = _load("libqcgpu.so")
        for name, (res, args) in _SIGS.items():
            if hasattr(l, name):
                f = getattr(l, name)
                f.restype = res
                f.argtypes = args
        _lib = l
    return _lib


def qsym_lib():
    """The drop-in libqsym.so exporting the reference's symAllowed symbol."""
    global _qsym
    if _qsym is None:
        q = _load("libqsym.so")
        q.symAllowed.restype = c_int
        q.symAllowed.argtypes = [c_int, c_int, c_vp, c_vp, c_vp] + [c_vp] * 8
        _qsym = q
    return _qsym


def ptr(a):
    """Address of a NumPy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, numpy.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def check(rc, what):
    if rc < 0:
        msg = lib().qc_last_error()
        cmsg = lib().qc_last_cuda_error()
        raise NativeError("%s failed (%d): %s %s" % (what, rc, msg.decode() if msg else "",
                                                   cmsg.decode() if cmsg else ""))
    return rc
