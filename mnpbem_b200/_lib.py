"""ctypes binding of ``libmnpbem_b200.so`` (declared in include/mnpbem_b200.h).

The library is built in-tree by ``mnpbem_b200/build.py``.  Loading fails
loudly: there is no CPU fallback for any entry point.
"""

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libmnpbem_b200.so')

_P = C.c_void_p
_I64 = C.c_int64
_I = C.c_int
_D = C.c_double

# name -> argtypes (restype int unless listed in _RESTYPE)
SIGNATURES = {
    'mnpb_version': [],
    'mnpb_last_error': [],
    'mnpb_launch_count': [],
    'mnpb_prof_begin': [],
    'mnpb_prof_end': [_I, _P, _P, _P],
    'mnpb_prof_dump': [C.c_char_p],
    'mnpb_refinematrix': [_I64, _I64, _P, _P, _P, _P, _D, _D, _I64, _P, _P, _P, _P],
    'mnpb_refine_coefficients': [_P, _I64, _P, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P,
                                 _P, _P, _P, _P, _P, _P],
    'mnpb_refine_finalize': [_P, _I64, _I64, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_closure_sums': [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_static_matrix': [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64],
    'mnpb_assemble_ret': [_P, _I64, _I64, _P, _P, _P, _I, _P, _P, _P, _I64, _P, _P, _P, _P, _I,
                          _P, _P, _P, _P, _I64, _I64, _I64],
    'mnpb_assemble_ret2': [_P, _I64, _I64, _P, _P, _P, _I, _P, _P, _P, _I64, _P, _P, _P, _P,
                           _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _I64],
    'mnpb_bemret_workspace_mixed': [_I64, _I64],
    'mnpb_bemret_init_mixed': [_P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, _P, _P, _I64],
    'mnpb_bemret_dinv_floats': [_I64, _I64],
    'mnpb_bemret_refine_workspace': [_I64, _I64, _I64],
    'mnpb_bemret_solve_refine': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _P, _P, _I, _D, _P, _P, _P, _I64],
    'mnpb_f32_workspace': [_I64, _I64],
    'mnpb_getrf_c32p': [_P, _I64, _I64, _P, _I64, _I64, _I64, _P, _I64, _P, _P, _I64],
    'mnpb_getri_c32p': [_P, _I64, _I64, _P, _I64, _I64, _I64, _P, _I64, _P, _I64, _I64, _I64,
                        _P, _I64],
    'mnpb_getrs_c32p': [_P, _I64, _I64, _I64, _P, _I64, _I64, _I64, _P, _I64, _P, _I64, _I64,
                        _I64, _P, _I64],
    'mnpb_bemret_workspace_f64': [_I64, _I64],
    'mnpb_bemret_init_f64': [_P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P, _I64],
    'mnpb_bemret_solve_f64': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _I64, _P, _P, _P, _I64],
    'mnpb_bemret_excitation': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _I64, _P],
    'mnpb_getrf_f64': [_P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P],
    'mnpb_getrs_f64': [_P, _I64, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _I64, _I64],
    'mnpb_zgemm': [_P, _I64, _I64, _I64, _I64, _D, _D, _P, _I64, _I64, _P, _I64, _I64, _D, _D,
                   _P, _I64, _I64],
    'mnpb_cgemm_tf32_workspace': [_I64, _I64, _I64],
    'mnpb_cgemm_tf32': [_P, _I64, _I64, _I64, _I64, C.c_float, _P, _I64, _I64, _I64, _P, _I64,
                        _I64, _I64, C.c_float, _P, _I64, _I64, _I64, _P, _I64],
    'mnpb_cgemm_tf32_ex': [_P, _I64, _I64, _I64, _I64, C.c_float, _P, _I64, _I64, _I64, _P,
                           _I64, _I64, _I64, C.c_float, _P, _I64, _I64, _I64, _P, _I64,
                           C.c_int32],
    'mnpb_cgemm_tf32_noalloc': [_P, _I64, _I64, _I64, _I64, C.c_float, _P, _I64, _I64, _I64,
                                _P, _I64, _I64, _I64, C.c_float, _P, _I64, _I64, _I64],
    'mnpb_tc_error': [_P, _P],
    'mnpb_gemm_config': [C.c_int32, C.c_int32, C.c_int32],
    'mnpb_gemm_config_mn': [C.c_int32],
    'mnpb_wait_probe': [_P, C.c_int32, _I64, _P],
    'mnpb_hmat_aca': [_P, _I64, _P, _I64, _P, _I64, _P, _P, _P, _I64, _I64, _D, _P, _P],
    'mnpb_hmat_gather_dense': [_P, _P, _I64, _P, _I64, _P, _P, _P],
    'mnpb_hmat_compact': [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_hmat_matvec': [_P, _I64, _I64, _I64, _P, _P, _I64, _I64, _P, _P, _I64, _P, _P, _P,
                         _I64, _P],
    'mnpb_bem_afun': [_P, _I64, _I64, _P, _P, _P, _P, _P, _D, _D, _D, _D, _D, _P],
    'mnpb_gmres_workspace': [_I64, _I64],
    'mnpb_gmres_arnoldi': [_P, _I64, _I64, _P, _I64, _P, _P, _P, _P, _I64],
    'mnpb_gmres_givens': [_P, _I64, _P, _I64, _P, _P, _P, _P],
    'mnpb_gmres_update': [_P, _I64, _I64, _P, _I64, _P, _P, _I64, _P, _P],
    'mnpb_vec_norms': [_P, _I64, _I64, _P, _I64, _P, _P],
    'mnpb_mlp_gemm': [_P, _I64, _I64, _I64, _P, _I64, _I64, _P, _I64, _I64, C.c_int32, _P, _I64,
                      _I64, _P, C.c_int32, _P, _I64, _P],
    'mnpb_mlp_silu_back': [_P, _I64, _P, _P, _P],
    'mnpb_mlp_colsum': [_P, _I64, _I64, _P, _I64, _P],
    'mnpb_mlp_mse': [_P, _I64, _P, _P, _P, _P],
    'mnpb_mlp_adam': [_P, _I64, _P, _P, _P, _P, _P, _D, _D, _D, _D, _I64],
    'mnpb_mlp_to_bf16': [_P, _I64, _P, _P],
    'mnpb_stat_matrix': [_P, _I64, _I64, _P, _I64, _P, _P, _I64, _I64],
    'mnpb_green_eval': [_P, _I64, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I64, _I64,
                        _P, _I64, _P],
    'mnpb_green_apply': [_P, _I64, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I64,
                         _P, _P],
    'mnpb_planewave_potential': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_farfield': [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_dipole_potential': [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P, _I, _P, _P,
                              _P, _P],
    'mnpb_dipole_field': [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P,
                          _P],
    'mnpb_dipole_farfield': [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_refine_points': [_P, _I64, _P, _I64, _P, _I64, _P, _P, _P, _P, _P, _P, _P],
    'mnpb_point_green': [_P, _I64, _P, _P, _I64, _P, _P, _P, _I, _P, _P, _P, _P, _P, _I, _I64,
                         _I64, _I64, _P, _P, _P, _P],
    'mnpb_eels_potential': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P,
                            _P, _D, _D, _P, _P, _P, _P],
    'mnpb_eels_infty': [_P, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _D, _D, _D,
                        _P, _P],
    'mnpb_eels_wire': [_P, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _I64, _P, _P,
                       _D, _D, _D, _P, _P, _P, _P],
    'mnpb_dipole_stat_field': [_P, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P],
    'mnpb_eels_field': [_P, _I64, _I64, _P, _P, _I, _P, _P, _D, _D, _P, _P, _P],
    'mnpb_pad_entries': [_P, _I64, _I64, _P, _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _I64,
                         _I64, _I64],
    'mnpb_mirror_contract': [_P, _I64, _I64, _I64, _I64, _P, _I64, _I64, _P, _P, _I64, _I64],
    'mnpb_bemret_mirror_workspace': [_I64, _I64],
    'mnpb_bemret_init_mirror_f64': [_P, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _P,
                                    _I64],
    'mnpb_bemret_sigma_mirror_f64': [_P, _I64, _I64, _I64, _P, _P, _P, _I64, _I64, _P, _P, _P,
                                     C.c_int32, C.c_int32, C.c_int32, _P, _I64, _P, _P],
    'mnpb_bemret_solve_mirror_workspace': [_I64, _I64, _I64],
    'mnpb_bemret_solve_mirror_f64': [_P, _I64, _I64, _I64, _I64, _P, _P, _P, _P, _I64, _I64, _P,
                                     _P, _I64, _P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P,
                                     _P, _P, _P, _I64],
    'mnpb_point_green_eval': [_P, _I64, _P, _P, _I64, _P, _P, _P, _I, _P, _P, _P, _P, _P, _I,
                              _I, _I64, _I64, _P],
}
_RESTYPE = {'mnpb_last_error': C.c_char_p, 'mnpb_launch_count': C.c_int64,
            'mnpb_cgemm_tf32_workspace': C.c_int64, 'mnpb_bemret_workspace_mixed': C.c_int64,
            'mnpb_bemret_mirror_workspace': C.c_int64,
            'mnpb_bemret_solve_mirror_workspace': C.c_int64,
            'mnpb_bemret_refine_workspace': C.c_int64, 'mnpb_f32_workspace': C.c_int64, 'mnpb_bemret_dinv_floats': C.c_int64,
            'mnpb_bemret_workspace_f64': C.c_int64, 'mnpb_gmres_workspace': C.c_int64}

_lib = None


class MNPBError(RuntimeError):
    """A library entry point returned a non-zero status."""

    def __init__(self, name, code, msg):
        super().__init__("{} failed (code {}): {}".format(name, code, msg))
        self.code = code


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("mnpbem_b200: {} is missing; build it with "
                              "`python -m mnpbem_b200.build`".format(LIB_PATH))
        h = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(h, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = h
    return _lib


def call(name, *args):
    """Call an entry point; raise MNPBError on a non-zero status."""
    fn = getattr(lib(), name)
    rc = fn(*args)
    if rc != 0:
        raise MNPBError(name, rc, lib().mnpb_last_error().decode(errors='replace'))
    return rc


def launch_count():
    return int(lib().mnpb_launch_count())


PROF_CLASSES = ['assemble', 'refine', 'zgemm_f64', 'lu_panel', 'trsm_small', 'swap',
                'elementwise', 'tc_gemm', 'farfield', 'sgemm_f32', 'matvec', 'trsv',
                'tc_pack', 'refine_elementwise', 'aca', 'hmat_matvec', 'gmres_arnoldi', 'mlp']


def prof_begin():
    call('mnpb_prof_begin')


def prof_end():
    """{class: (ms, work, launches)} for the launches since prof_begin()."""
    import numpy as np
    n = 24
    ms = np.zeros(n)
    work = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int64)
    call('mnpb_prof_end', n, ptr(ms), ptr(work), ptr(cnt))
    out = {}
    for i in range(n):
        if cnt[i]:
            name = PROF_CLASSES[i] if i < len(PROF_CLASSES) else 'class%d' % i
            out[name] = (float(ms[i]), float(work[i]), int(cnt[i]))
    return out


class _Ref(object):
    """Pointer argument that keeps its tensor/array alive until the call has
    been issued (a temporary freed earlier could hand its memory to the next
    temporary of the same call).  After the launch, stream ordering makes the
    memory safe to reuse."""

    __slots__ = ('obj', '_as_parameter_')

    def __init__(self, obj, addr):
        self.obj = obj
        self._as_parameter_ = C.c_void_p(addr)


def ptr(t):
    """Device/host address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, 'data_ptr'):
        if not t.is_contiguous():
            raise ValueError("ptr: tensor must be contiguous")
        return _Ref(t, t.data_ptr())
    if not t.flags['C_CONTIGUOUS']:
        raise ValueError("ptr: array must be C-contiguous")
    return _Ref(t, t.ctypes.data)


def stream_handle(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)
