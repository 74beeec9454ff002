"""blasfeo_b200: BLASFEO's level-3 / LAPACK hot path on NVIDIA B200 (sm_100a).

The product is the C-ABI shared library ``libblasfeo_b200.so`` (declared in
``include/blasfeo_b200.h``).  This module loads it with ctypes and mirrors the
reference's BLASFEO API for Python callers: the same routine names and
argument meanings (``blasfeo_dgemm_nt(m, n, k, alpha, sA, ai, aj, ...)``),
with matrices that live in device memory.

Device memory is plain CUDA memory; torch is used only to allocate it and to
provide streams.  Loading fails loudly when the shared library is missing:
there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libblasfeo_b200.so")


class BlasfeoError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise BlasfeoError("libblasfeo_b200.so not built: run `python blasfeo_b200/build.py` (%s)" % LIB_PATH)
    return C.CDLL(LIB_PATH)


lib = _load()


class dmat(C.Structure):
    """struct blasfeo_dmat (include/blasfeo_common.h:67-80 layout)."""
    _fields_ = [("mem", C.c_void_p), ("pA", C.c_void_p), ("dA", C.c_void_p),
                ("m", C.c_int), ("n", C.c_int), ("pm", C.c_int), ("cn", C.c_int),
                ("use_dA", C.c_int), ("memsize", C.c_int)]


class smat(dmat):
    """struct blasfeo_smat (same layout as blasfeo_dmat, float pointers)."""


class dvec(C.Structure):
    _fields_ = [("mem", C.c_void_p), ("pa", C.c_void_p), ("m", C.c_int), ("pm", C.c_int),
                ("memsize", C.c_int)]


class svec(dvec):
    pass


class dmat_batch(C.Structure):
    _fields_ = [("mem", C.c_void_p), ("pA", C.c_void_p), ("dA", C.c_void_p),
                ("m", C.c_int), ("n", C.c_int), ("pm", C.c_int), ("cn", C.c_int),
                ("use_dA", C.c_int), ("batch", C.c_int), ("stride", C.c_longlong),
                ("memsize", C.c_size_t)]


class smat_batch(dmat_batch):
    pass


class dmat_batch_il(C.Structure):
    """struct blasfeo_dmat_batch_il (batch-interleaved slab)."""
    _fields_ = [("mem", C.c_void_p), ("m", C.c_int), ("n", C.c_int), ("pm", C.c_int), ("cn", C.c_int),
                ("batch", C.c_int), ("il", C.c_int), ("gstride", C.c_longlong), ("memsize", C.c_size_t)]


class cm_dmat(C.Structure):
    """struct blasfeo_cm_dmat (include/blasfeo_common.h:220-229 layout): pA is
    column-major with leading dimension m."""
    _fields_ = [("mem", C.c_void_p), ("pA", C.c_void_p), ("dA", C.c_void_p),
                ("m", C.c_int), ("n", C.c_int), ("use_dA", C.c_int), ("memsize", C.c_int)]


class cm_smat(cm_dmat):
    """struct blasfeo_cm_smat (same layout, float pointers)."""


P = C.POINTER
_i, _d, _f, _vp, _sz = C.c_int, C.c_double, C.c_float, C.c_void_p, C.c_size_t
_DM, _SM, _DV, _SV = P(dmat), P(smat), P(dvec), P(svec)
_DB, _SB = P(dmat_batch), P(smat_batch)


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


def _gemm_args(M, R):
    return [_i, _i, _i, R, M, _i, _i, M, _i, _i, R, M, _i, _i, M, _i, _i]


def _syrk_args(M, R):
    return [_i, _i, R, M, _i, _i, M, _i, _i, R, M, _i, _i, M, _i, _i]


def _trsm_args(M, R):
    return [_i, _i, R, M, _i, _i, M, _i, _i, M, _i, _i]


# ---- declarations (mirror include/blasfeo_b200.h) ----
_sig("blasfeo_b200_last_error", _i)
_sig("blasfeo_b200_error_string", C.c_char_p, _i)
_sig("blasfeo_b200_set_stream", None, _vp)
_sig("blasfeo_b200_get_stream", _vp)
_sig("blasfeo_b200_set_sync", None, _i)
_sig("blasfeo_b200_set_posv_engine", _i, _i)
_sig("blasfeo_b200_get_posv_engine", _i)
_sig("blasfeo_b200_version", _i)
_sig("blasfeo_b200_measure_fma_peak", _d, C.c_char, _i)
_sig("blasfeo_b200_set_wait_limit", None, C.c_uint)
_sig("blasfeo_b200_get_wait_limit", C.c_uint)
_sig("blasfeo_b200_check_wait_timeout", _i, _vp, _vp)
for p, M, V, R in (("d", _DM, _DV, _d), ("s", _SM, _SV, _f)):
    _sig("blasfeo_memsize_%smat" % p, _sz, _i, _i)
    _sig("blasfeo_memsize_diag_%smat" % p, _sz, _i, _i)
    _sig("blasfeo_create_%smat" % p, None, _i, _i, M, _vp)
    _sig("blasfeo_memsize_%svec" % p, _sz, _i)
    _sig("blasfeo_create_%svec" % p, None, _i, V, _vp)
    _sig("blasfeo_pack_%smat" % p, None, _i, _i, _vp, _i, M, _i, _i)
    _sig("blasfeo_unpack_%smat" % p, None, _i, _i, M, _i, _i, _vp, _i)
    _sig("blasfeo_pack_%svec" % p, None, _i, _vp, _i, V, _i)
    _sig("blasfeo_unpack_%svec" % p, None, _i, V, _i, _vp, _i)
    _sig("blasfeo_pack_tran_%smat" % p, None, _i, _i, _vp, _i, M, _i, _i)
    _sig("blasfeo_unpack_tran_%smat" % p, None, _i, _i, M, _i, _i, _vp, _i)
    _sig("blasfeo_%sgecp" % p, None, _i, _i, M, _i, _i, M, _i, _i)
    _sig("blasfeo_%sdiare" % p, None, _i, R, M, _i, _i)
    _sig("blasfeo_%srowsw" % p, None, _i, M, _i, _i, M, _i, _i)
    _sig("blasfeo_%sgemm_nt" % p, None, *_gemm_args(M, R))
    _sig("blasfeo_%ssyrk_ln" % p, None, *_syrk_args(M, R))
    _sig("blasfeo_%strsm_rltn" % p, None, *_trsm_args(M, R))
    _sig("blasfeo_%strmm_rlnn" % p, None, *_trsm_args(M, R))
    _sig("blasfeo_%spotrf_l" % p, None, _i, M, _i, _i, M, _i, _i)
    _sig("blasfeo_%ssyrk_%spotrf_ln" % (p, p), None, _i, _i, M, _i, _i, M, _i, _i, M, _i, _i, M, _i, _i)
    _sig("blasfeo_%sgetrf_rp" % p, None, _i, _i, M, _i, _i, M, _i, _i, P(_i))
    _sig("blasfeo_%sgeqrf_worksize" % p, _i, _i, _i)
    _sig("blasfeo_%sgeqrf" % p, None, _i, _i, M, _i, _i, M, _i, _i, _vp)
    _sig("blasfeo_%ssyrk_ln_mn" % p, None, _i, *_syrk_args(M, R))
    _sig("blasfeo_%strsm_rltu" % p, None, *_trsm_args(M, R))
    _sig("blasfeo_%spotrf_l_mn" % p, None, _i, _i, M, _i, _i, M, _i, _i)
    _sig("blasfeo_%sgetrf_np" % p, None, _i, _i, M, _i, _i, M, _i, _i)
for p, R, M in (("d", _d, P(cm_dmat)), ("s", _f, P(cm_smat))):
    _sig("blasfeo_cm_memsize_%smat" % p, _sz, _i, _i)
    _sig("blasfeo_cm_create_%smat" % p, None, _i, _i, M, _vp)
    _sig("blasfeo_cm_%sgemm_nt" % p, None, *_gemm_args(M, R))
    _sig("blasfeo_cm_%strsm_rltn" % p, None, *_trsm_args(M, R))
    _sig("blasfeo_cm_%spotrf_l" % p, None, _i, M, _i, _i, M, _i, _i)
_sig("blasfeo_cm_dsyrk_ln", None, *_syrk_args(P(cm_dmat), _d))
_sig("blasfeo_cm_dgetrf_rp", None, _i, _i, P(cm_dmat), _i, _i, P(cm_dmat), _i, _i, P(_i))
_sig("blasfeo_dgemv_n", None, _i, _i, _d, _DM, _i, _i, _DV, _i, _d, _DV, _i, _DV, _i)
_sig("blasfeo_dtrsv_lnn", None, _i, _DM, _i, _i, _DV, _i, _DV, _i)
_sig("blasfeo_dtrsv_ltn", None, _i, _DM, _i, _i, _DV, _i, _DV, _i)
for p, B, R, M in (("d", _DB, _d, _DM), ("s", _SB, _f, _SM)):
    _sig("blasfeo_memsize_%smat_batch" % p, _sz, _i, _i, _i)
    _sig("blasfeo_create_%smat_batch" % p, None, _i, _i, _i, B, _vp)
    _sig("blasfeo_%smat_batch_instance" % p, None, B, _i, M)
    _sig("blasfeo_pack_%smat_batch" % p, _i, _i, _i, _i, _vp, _i, C.c_longlong, B, _i, _i, _vp)
    _sig("blasfeo_unpack_%smat_batch" % p, _i, _i, _i, _i, B, _i, _i, _vp, _i, C.c_longlong, _vp)
    _sig("blasfeo_%sgemm_nt_batch" % p, _i, _i, *(_gemm_args(B, R) + [_vp]))
    _sig("blasfeo_%ssyrk_ln_batch" % p, _i, _i, *(_syrk_args(B, R) + [_vp]))
    _sig("blasfeo_%strsm_rltn_batch" % p, _i, _i, *(_trsm_args(B, R) + [_vp]))
    _sig("blasfeo_%spotrf_l_batch" % p, _i, _i, _i, B, _i, _i, B, _i, _i, _vp, _vp)
    _sig("blasfeo_%ssyrk_%spotrf_ln_batch" % (p, p), _i, _i, _i, _i, B, _i, _i, B, _i, _i, B, _i, _i, B, _i, _i,
         _vp, _vp)
    _sig("blasfeo_%sgetrf_rp_batch" % p, _i, _i, _i, _i, B, _i, _i, B, _i, _i, _vp, _vp, _vp)
    _sig("blasfeo_%sgeqrf_batch" % p, _i, _i, _i, _i, B, _i, _i, B, _i, _i, _vp)
    _sig("blasfeo_%ssyrk_ln_mn_batch" % p, _i, _i, _i, *(_syrk_args(B, R) + [_vp]))
    _sig("blasfeo_%strsm_rltu_batch" % p, _i, _i, *(_trsm_args(B, R) + [_vp]))
    _sig("blasfeo_%spotrf_l_mn_batch" % p, _i, _i, _i, _i, B, _i, _i, B, _i, _i, _vp, _vp)
    _sig("blasfeo_%sgetrf_np_batch" % p, _i, _i, _i, _i, B, _i, _i, B, _i, _i, _vp, _vp)
_sig("blasfeo_dgemm_nt_vbatch", _i, _i, _vp, _vp, _vp, _i, _i, _i, _d, _vp, _vp, _d, _vp, _vp, _vp)
_sig("blasfeo_dpotrf_l_vbatch", _i, _i, _vp, _i, _vp, _vp, _vp, _vp)
_sig("blasfeo_dgetrf_rp_vbatch", _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _i, _vp, _vp)
_sig("blasfeo_dgeqrf_vbatch", _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp)
_sig("blasfeo_b200_num_variants", _i, _i)
_sig("blasfeo_dgemm_nt_vbatch_variant", _i, _i, _vp, _vp, _vp, _i, _i, _i, _d, _vp, _vp, _d, _vp, _vp, _i, _vp)
_sig("blasfeo_dpotrf_l_vbatch_variant", _i, _i, _vp, _i, _vp, _vp, _vp, _i, _vp)
_sig("blasfeo_dgetrf_rp_vbatch_variant", _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _i, _vp, _i, _vp)
_sig("blasfeo_dgeqrf_vbatch_variant", _i, _i, _vp, _vp, _i, _i, _vp, _vp, _i, _vp)
_sig("blasfeo_dposv_worksize", _sz, _i)
_sig("blasfeo_dposv_worksize_n", _sz, _i, _i, _i)
_sig("blasfeo_dposv_l_vbatch", _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _sz, _vp)
_sig("blasfeo_dsposv_l_vbatch", _i, _i, _vp, _i, _vp, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp, _sz, _vp)
_sig("blasfeo_dsposv_l_vbatch_mapped", _i, _i, _vp, _i, _vp, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp, _sz, _vp)
_sig("blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch", _i, _i, _i, _i, _d, _DB, _DB, _DB, _DB, _DB, _DB, _DB, _vp, _vp)
_sig("blasfeo_dric_trf_batch", _i, _i, _i, _i, _i, _DB, _DB, _DB, _vp, _vp)
_sig("blasfeo_sric_trf_batch", _i, _i, _i, _i, _i, _SB, _SB, _SB, _vp, _vp)
_LL = C.c_longlong
_sig("blasfeo_dric_trs_batch", _i, _i, _i, _i, _i, _DB, _DB, _vp, _LL, _vp, _LL, _vp, _LL, _vp, _LL, _vp)
_sig("blasfeo_dric_gains_batch", _i, _i, _i, _i, _i, _DB, _DB, _vp)
_sig("blasfeo_dsric_sv_worksize", _sz, _i, _i, _i)
_sig("blasfeo_dsric_sv_batch", _i, _i, _i, _i, _i, _DB, _DB, _vp, _LL, _vp, _LL, _vp, _LL, _vp, _LL, _i, _d, _vp, _vp,
     _vp, _vp, _sz, _vp)
_sig("blasfeo_b200_mlp_param_count", _i, _i, _i)
_sig("blasfeo_b200_mlp_work_bytes", _sz, _i, _i)
_sig("blasfeo_b200_mlp_forward", _i, _i, _i, _vp, _i, _vp, _vp, _vp, _vp)
_sig("blasfeo_b200_mlp_grad", _i, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp)
_sig("blasfeo_b200_mlp_adam", _i, _i, _vp, _vp, _vp, _vp, _i, _f, _vp)
_sig("blasfeo_b200_cost_model_nfeat", _i)
_IL = P(dmat_batch_il)
_sig("blasfeo_memsize_dmat_batch_il", _sz, _i, _i, _i)
_sig("blasfeo_create_dmat_batch_il", None, _i, _i, _i, _IL, _vp)
_sig("blasfeo_dmat_batch_to_il", _i, _DB, _IL, _vp)
_sig("blasfeo_dmat_batch_from_il", _i, _IL, _DB, _vp)
_sig("blasfeo_pack_dmat_batch_il", _i, _i, _i, _i, _vp, _i, C.c_longlong, _IL, _vp)
_sig("blasfeo_unpack_dmat_batch_il", _i, _i, _i, _i, _IL, _vp, _i, C.c_longlong, _vp)
_sig("blasfeo_dpotrf_l_batch_il", _i, _i, _i, _IL, _IL, _vp, _vp)
_sig("blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il", _i, _i, _i, _i, _d, _IL, _IL, _IL, _IL, _IL, _IL, _IL, _vp, _vp)
_sig("blasfeo_dric_trf_batch_il", _i, _i, _i, _i, _i, _IL, _IL, _IL, _vp, _vp)
_sig("blasfeo_b200_set_cost_model", _i, _i, _i, _vp)
_sig("blasfeo_b200_clear_cost_model", None)
_sig("blasfeo_b200_dispatch_pick", _i, _i, _i, _vp, _vp, _vp, _i, _i, _i, _vp)
_sig("blasfeo_dsposv_noalloc_scratch_bytes", _sz)
_sig("blasfeo_dsposv_l_vbatch_noalloc", _i, _i, _vp, _i, _vp, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp)


def check(status=None):
    """Raise on a non-zero status (or on the recorded last error)."""
    if status is None:
        status = lib.blasfeo_b200_last_error()
    if status:
        raise BlasfeoError("blasfeo_b200: %s (%d)" % (lib.blasfeo_b200_error_string(status).decode(), status))


from .api import *  # noqa: E402,F401,F403
