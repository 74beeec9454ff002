"""CPU tests of the C-ABI boundary: the shared library loads, exports every
function declared in include/blasfeo_b200.h, keeps the reference's descriptor
layout and storage sizes, and rejects bad arguments before touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "blasfeo_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(blasfeo_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_hot_path():
    names = declared_functions()
    for r in ["blasfeo_dgemm_nt", "blasfeo_dsyrk_ln", "blasfeo_dtrsm_rltn", "blasfeo_dpotrf_l", "blasfeo_dgetrf_rp",
              "blasfeo_dgeqrf", "blasfeo_dgeqrf_worksize", "blasfeo_dsyrk_dpotrf_ln", "blasfeo_sgemm_nt",
              "blasfeo_ssyrk_ln", "blasfeo_strsm_rltn", "blasfeo_spotrf_l", "blasfeo_sgetrf_rp", "blasfeo_sgeqrf",
              "blasfeo_memsize_dmat", "blasfeo_create_dmat", "blasfeo_pack_dmat", "blasfeo_unpack_dmat"]:
        assert r in names, r


def test_library_exports_every_declared_symbol():
    import blasfeo_b200
    missing = [n for n in declared_functions() if not hasattr(blasfeo_b200.lib, n)]
    assert not missing, missing


def test_descriptor_layout():
    import blasfeo_b200 as bf
    assert C.sizeof(bf.dmat) == 48 and C.sizeof(bf.dvec) == 32
    assert [f for f, _ in bf.dmat._fields_] == ["mem", "pA", "dA", "m", "n", "pm", "cn", "use_dA", "memsize"]


@pytest.mark.parametrize("mn", [(64, 64), (16, 16), (16, 32), (5, 3), (1, 1), (257, 13), (13, 257)])
def test_memsize_and_create_match_reference(mn):
    import blasfeo_b200 as bf
    m, n = mn
    pm, cn = (m + 3) // 4 * 4, (n + 3) // 4 * 4
    dl = (min(m, n) + 15) // 16 * 16
    want = ((pm * cn + dl) * 8 + 63) // 64 * 64
    assert bf.lib.blasfeo_memsize_dmat(m, n) == want
    s = bf.dmat()
    base = 0x10000
    bf.lib.blasfeo_create_dmat(m, n, C.byref(s), C.c_void_p(base))
    assert (s.m, s.n, s.pm, s.cn, s.use_dA) == (m, n, pm, cn, 0)
    assert s.pA == base and s.dA == base + pm * cn * 8 and s.memsize == want
    from oracle.pyoracle import ref_available, ref_lib
    if ref_available("generic"):
        r = ref_lib("generic")
        r.blasfeo_memsize_dmat.restype = C.c_size_t
        assert r.blasfeo_memsize_dmat(m, n) == want
        r.blasfeo_memsize_smat.restype = C.c_size_t
        assert r.blasfeo_memsize_smat(m, n) == bf.lib.blasfeo_memsize_smat(m, n)


def test_batch_slab_layout():
    import blasfeo_b200 as bf
    s = bf.dmat_batch()
    bf.lib.blasfeo_create_dmat_batch(16, 16, 100, C.byref(s), C.c_void_p(0x1000))
    assert s.stride * 8 == bf.lib.blasfeo_memsize_dmat(16, 16)
    assert s.memsize == 100 * bf.lib.blasfeo_memsize_dmat(16, 16)
    inst = bf.dmat()
    bf.lib.blasfeo_dmat_batch_instance(C.byref(s), 7, C.byref(inst))
    assert inst.pA == 0x1000 + 7 * s.stride * 8


def test_bad_arguments_rejected_without_gpu():
    import blasfeo_b200 as bf
    lib = bf.lib
    EINVAL = 1
    s = bf.dmat_batch()
    assert lib.blasfeo_dgemm_nt_batch(-1, 4, 4, 4, 1.0, None, 0, 0, None, 0, 0, 0.0, None, 0, 0, None, 0, 0, None) == EINVAL
    assert lib.blasfeo_dpotrf_l_batch(4, 4, None, 0, 0, C.byref(s), 0, 0, None, None) == EINVAL
    assert lib.blasfeo_dposv_l_vbatch(-1, None, 4, None, None, None, None, None, 0, None) == EINVAL
    assert lib.blasfeo_dsposv_l_vbatch(3, None, 4, None, None, None, 10, 1e-12, None, None, None, None, 0, None) == EINVAL
    # zero-size calls are no-ops that succeed
    assert lib.blasfeo_dpotrf_l_batch(0, 4, C.byref(s), 0, 0, C.byref(s), 0, 0, None, None) == 0
    assert lib.blasfeo_dgeqrf_worksize(12, 8) == 4 * (12 + 8) * 8


def test_error_strings():
    import blasfeo_b200 as bf
    assert bf.lib.blasfeo_b200_error_string(0) == b"ok"
    assert b"invalid" in bf.lib.blasfeo_b200_error_string(1)


def test_cm_descriptor_layout():
    import blasfeo_b200 as bf
    assert C.sizeof(bf.cm_dmat) == 40 and C.sizeof(bf.cm_smat) == 40
    assert [f for f, _ in bf.cm_dmat._fields_] == ["mem", "pA", "dA", "m", "n", "use_dA", "memsize"]


@pytest.mark.parametrize("mn", [(64, 64), (5, 3), (3, 5), (1, 1), (257, 13)])
def test_cm_memsize_and_create_match_reference(mn):
    """blasfeo_cm_memsize_dmat / blasfeo_cm_create_dmat (auxiliary/d_aux_common.c:111,121):
    m*n elements then min(m,n) for dA, no rounding."""
    import blasfeo_b200 as bf
    m, n = mn
    want = (m * n + min(m, n)) * 8
    assert bf.lib.blasfeo_cm_memsize_dmat(m, n) == want
    assert bf.lib.blasfeo_cm_memsize_smat(m, n) == want // 2
    s = bf.cm_dmat()
    base = 0x20000
    bf.lib.blasfeo_cm_create_dmat(m, n, C.byref(s), C.c_void_p(base))
    assert (s.m, s.n, s.use_dA, s.memsize) == (m, n, 0, want)
    assert s.mem == base and s.pA == base and s.dA == base + m * n * 8
    from oracle.pyoracle import ref_available, ref_lib
    if ref_available("generic"):
        r = ref_lib("generic")
        r.blasfeo_cm_memsize_dmat.restype = C.c_size_t
        assert r.blasfeo_cm_memsize_dmat(m, n) == want
        # the reference's create takes a struct blasfeo_pm_dmat pointer
        # (include/blasfeo_d_aux.h:237; include/blasfeo_common.h:173-185: mem,
        # pA, dA, m, n, pm, cn, use_dA, ps, memsize): read its fields there
        raw = (C.c_ubyte * 64)()
        r.blasfeo_cm_create_dmat(m, n, raw, C.c_void_p(base))
        b = bytes(raw)
        q = lambda off: int.from_bytes(b[off:off + 8], "little")
        i = lambda off: int.from_bytes(b[off:off + 4], "little", signed=True)
        assert (q(8), q(16), i(24), i(28), i(40), i(48)) == (s.pA, s.dA, s.m, s.n, s.use_dA, s.memsize)


def test_cm_bad_arguments_rejected_without_gpu():
    """The column-major entry points check their descriptors before any device
    work: a NULL descriptor or pA records EINVAL; empty sizes are no-ops."""
    import blasfeo_b200 as bf
    lib = bf.lib
    EINVAL = 1
    lib.blasfeo_b200_last_error()  # clear
    good = bf.cm_dmat()
    lib.blasfeo_cm_create_dmat(8, 8, C.byref(good), C.c_void_p(0x3000))
    empty = bf.cm_dmat()  # pA NULL
    lib.blasfeo_cm_dpotrf_l(8, None, 0, 0, C.byref(good), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    lib.blasfeo_cm_dpotrf_l(8, C.byref(empty), 0, 0, C.byref(good), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    lib.blasfeo_cm_dgemm_nt(4, 4, -1, 1.0, C.byref(good), 0, 0, C.byref(good), 0, 0, 0.0, C.byref(good), 0, 0,
                            C.byref(good), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    lib.blasfeo_cm_dgetrf_rp(4, 4, C.byref(good), 0, 0, C.byref(good), 0, 0, None)
    assert lib.blasfeo_b200_last_error() == EINVAL
    s = bf.cm_smat()
    lib.blasfeo_cm_strsm_rltn(4, 4, 1.0, None, 0, 0, C.byref(s), 0, 0, C.byref(s), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    # empty sizes: nothing happens, nothing is recorded
    lib.blasfeo_cm_dpotrf_l(0, None, 0, 0, None, 0, 0)
    lib.blasfeo_cm_dgemm_nt(0, 4, 4, 1.0, None, 0, 0, None, 0, 0, 0.0, None, 0, 0, None, 0, 0)
    assert lib.blasfeo_b200_last_error() == 0


def test_cm_out_of_range_blocks_rejected_without_gpu():
    """Every operand block of the column-major entry points must lie inside its
    descriptor's m x n matrix (m is the leading dimension): a negative offset
    or a block that runs past the last row or column records EINVAL before any
    staging kernel could read or write outside the caller's buffer."""
    import blasfeo_b200 as bf
    lib = bf.lib
    EINVAL = 1
    lib.blasfeo_b200_last_error()  # clear
    a = bf.cm_dmat()
    lib.blasfeo_cm_create_dmat(8, 6, C.byref(a), C.c_void_p(0x3000))
    A = C.byref(a)
    bad_calls = [
        # gemm_nt: A m x k at (ai, aj), B n x k, C and D m x n
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, -1, 0, A, 0, 0, 0.0, A, 0, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, 5, 0, A, 0, 0, 0.0, A, 0, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, 0, 3, A, 0, 0, 0.0, A, 0, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, 0, 0, A, 0, -2, 0.0, A, 0, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, 0, 0, A, 0, 0, 1.0, A, 6, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dgemm_nt(4, 4, 4, 1.0, A, 0, 0, A, 0, 0, 0.0, A, 0, 0, A, 0, 3),
        lambda: lib.blasfeo_cm_dgemm_nt(9, 4, 4, 1.0, A, 0, 0, A, 0, 0, 0.0, A, 0, 0, A, 0, 0),
        # syrk_ln: D m x m
        lambda: lib.blasfeo_cm_dsyrk_ln(7, 2, 1.0, A, 0, 0, A, 0, 0, 0.0, A, 0, 0, A, 0, 0),
        # trsm_rltn: A n x n, B and D m x n
        lambda: lib.blasfeo_cm_dtrsm_rltn(4, 6, 1.0, A, 3, 0, A, 0, 0, A, 0, 0),
        lambda: lib.blasfeo_cm_dtrsm_rltn(4, 4, 1.0, A, 0, 0, A, 0, 0, A, 0, -1),
        # potrf_l: m x m
        lambda: lib.blasfeo_cm_dpotrf_l(6, A, 0, 1, A, 0, 0),
        lambda: lib.blasfeo_cm_dpotrf_l(6, A, 0, 0, A, 3, 0),
        # getrf_rp: m x n
        lambda: lib.blasfeo_cm_dgetrf_rp(8, 6, A, 1, 0, A, 0, 0, (C.c_int * 8)()),
        lambda: lib.blasfeo_cm_dgetrf_rp(8, 7, A, 0, 0, A, 0, 0, (C.c_int * 8)()),
    ]
    for i, call in enumerate(bad_calls):
        call()
        assert lib.blasfeo_b200_last_error() == EINVAL, i
    s = bf.cm_smat()
    lib.blasfeo_cm_create_smat(8, 6, C.byref(s), C.c_void_p(0x3000))
    lib.blasfeo_cm_strsm_rltn(4, 6, 1.0, C.byref(s), 3, 0, C.byref(s), 0, 0, C.byref(s), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    lib.blasfeo_cm_spotrf_l(7, C.byref(s), 0, 0, C.byref(s), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL
    lib.blasfeo_cm_sgemm_nt(4, 4, 7, 1.0, C.byref(s), 0, 0, C.byref(s), 0, 0, 0.0, C.byref(s), 0, 0, C.byref(s), 0, 0)
    assert lib.blasfeo_b200_last_error() == EINVAL


def test_wait_limit_setting():
    import blasfeo_b200 as bf
    lib = bf.lib
    default = lib.blasfeo_b200_get_wait_limit()
    assert default == 1 << 24
    lib.blasfeo_b200_set_wait_limit(1000)
    assert lib.blasfeo_b200_get_wait_limit() == 1000
    lib.blasfeo_b200_set_wait_limit(0)
    assert lib.blasfeo_b200_get_wait_limit() == default
    assert lib.blasfeo_b200_check_wait_timeout(None, None) == 1
