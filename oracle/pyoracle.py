"""ctypes access to the CPU oracle and to the compiled reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker; the product package
``blasfeo_b200`` never imports it.

Two libraries share one calling convention (the BLASFEO panel-major C API with
``struct blasfeo_dmat`` / ``struct blasfeo_smat`` descriptors in host memory):

* ``liboracle.so``  - the plain-C restatement in oracle.c / oracle_x.h
  (symbols ``oracle_d_*`` / ``oracle_s_*``);
* ``_ref/libblasfeo_ref_{generic,haswell}.so`` - BLASFEO 0.1.4.2 compiled from
  its own sources by oracle/Makefile (symbols ``blasfeo_*`` for the HP panel-major
  path and ``blasfeo_ref_*`` for its REFERENCE backend);
* ``_ref/libblasfeo_ref_cm_generic.so`` - the GENERIC build plus the reference's
  column-major ``blasfeo_cm_d*`` routines (blasfeo_hp_cm/, BLAS_API).

Host matrices are numpy arrays in column-major order; :class:`HostMat` packs
them into panel-major storage (panel size 4) owned by a numpy buffer.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class DMat(C.Structure):
    _fields_ = [("mem", C.c_void_p), ("pA", C.c_void_p), ("dA", C.c_void_p),
                ("m", C.c_int), ("n", C.c_int), ("pm", C.c_int), ("cn", C.c_int),
                ("use_dA", C.c_int), ("memsize", C.c_int)]


class DVec(C.Structure):
    _fields_ = [("mem", C.c_void_p), ("pa", C.c_void_p), ("m", C.c_int), ("pm", C.c_int),
                ("memsize", C.c_int)]


def _lib(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path)


def oracle_lib():
    return _lib(os.path.join(HERE, "liboracle.so"))


def ref_lib(target="generic"):
    return _lib(os.path.join(HERE, "_ref", "libblasfeo_ref_%s.so" % target))


def ref_cm_lib():
    """The GENERIC build plus the reference's column-major blasfeo_cm_d* routines."""
    return _lib(os.path.join(HERE, "_ref", "libblasfeo_ref_cm_generic.so"))


def ref_cm_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libblasfeo_ref_cm_generic.so"))


class CmDMat(C.Structure):
    """struct blasfeo_cm_dmat (include/blasfeo_common.h:220-229)."""
    _fields_ = [("mem", C.c_void_p), ("pA", C.c_void_p), ("dA", C.c_void_p),
                ("m", C.c_int), ("n", C.c_int), ("use_dA", C.c_int), ("memsize", C.c_int)]


class HostCmMat:
    """A column-major host matrix (leading dimension m) with a cm descriptor
    (struct blasfeo_cm_dmat, or blasfeo_cm_smat for float32: same layout)."""

    def __init__(self, data, dtype=np.float64):
        self.a = np.asfortranarray(np.array(data, dtype=dtype))
        self.m, self.n = self.a.shape
        self.dA = np.zeros(max(self.m, self.n) + 8, dtype=dtype)
        self.desc = CmDMat()
        self.desc.mem = self.desc.pA = self.a.ctypes.data
        self.desc.dA = self.dA.ctypes.data
        self.desc.m, self.desc.n = self.m, self.n

    @property
    def ref(self):
        return C.byref(self.desc)


def ref_available(target="generic"):
    return os.path.exists(os.path.join(HERE, "_ref", "libblasfeo_ref_%s.so" % target))


def ps_of(dtype, target="generic"):
    """Panel size of the layout: 4 everywhere except single precision on Haswell (8)."""
    if np.dtype(dtype) == np.float32 and target == "haswell":
        return 8
    return 4


def _aligned_zeros(nel, dtype, align=64):
    """Zeroed numpy array whose data pointer is ``align``-byte aligned (the HP
    kernels use aligned vector loads, as blasfeo_malloc_align guarantees)."""
    dtype = np.dtype(dtype)
    raw = np.zeros(nel * dtype.itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + nel * dtype.itemsize].view(dtype)


class HostMat:
    """A panel-major matrix in host memory with a BLASFEO-style descriptor."""

    def __init__(self, m, n, dtype=np.float64, ps=4):
        self.m, self.n, self.ps = m, n, ps
        self.dtype = np.dtype(dtype)
        pm = (m + ps - 1) // ps * ps
        cn = (n + 3) // 4 * 4
        mn = min(m, n)
        al = ps * 4
        dl = (mn + al - 1) // al * al
        nel = pm * cn + dl
        self.buf = _aligned_zeros(nel, self.dtype)
        self.desc = DMat()
        self.desc.mem = self.buf.ctypes.data
        self.desc.pA = self.buf.ctypes.data
        self.desc.dA = self.buf.ctypes.data + pm * cn * self.dtype.itemsize
        self.desc.m, self.desc.n, self.desc.pm, self.desc.cn = m, n, pm, cn
        self.desc.use_dA = 0
        self.desc.memsize = (pm * cn + dl) * self.dtype.itemsize
        self.pm, self.cn = pm, cn

    def _idx(self, i, j):
        ps = self.ps
        return (i - i % ps) * self.cn + j * ps + i % ps

    def set(self, A, ai=0, aj=0):
        A = np.asarray(A, dtype=self.dtype)
        mm, nn = A.shape
        ii, jj = np.meshgrid(np.arange(mm) + ai, np.arange(nn) + aj, indexing="ij")
        self.buf[self._idx(ii, jj)] = A
        self.desc.use_dA = 0
        return self

    def get(self, m=None, n=None, ai=0, aj=0):
        m = self.m - ai if m is None else m
        n = self.n - aj if n is None else n
        ii, jj = np.meshgrid(np.arange(m) + ai, np.arange(n) + aj, indexing="ij")
        return self.buf[self._idx(ii, jj)].copy()

    def panel(self):
        """The raw panel-major array (pm*cn elements)."""
        return self.buf[: self.pm * self.cn]

    def diag(self, k=None):
        k = min(self.m, self.n) if k is None else k
        off = self.pm * self.cn
        return self.buf[off:off + k].copy()

    @property
    def ref(self):
        return C.byref(self.desc)


class HostVec:
    def __init__(self, m, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        self.buf = _aligned_zeros((m + 3) // 4 * 4 + 8, self.dtype)
        self.desc = DVec()
        self.desc.mem = self.buf.ctypes.data
        self.desc.pa = self.buf.ctypes.data
        self.desc.m = m
        self.desc.pm = (m + 3) // 4 * 4
        self.desc.memsize = self.desc.pm * self.dtype.itemsize
        self.m = m

    def set(self, x):
        self.buf[: len(x)] = x
        return self

    def get(self):
        return self.buf[: self.m].copy()

    @property
    def ref(self):
        return C.byref(self.desc)


class Api:
    """Uniform call surface over the oracle and the compiled reference.

    ``Api("oracle")`` -> liboracle.so; ``Api("hp", target)`` -> the compiled HP
    panel-major routines ``blasfeo_*``; ``Api("ref", target)`` -> the compiled
    REFERENCE backend ``blasfeo_ref_*``.
    """

    def __init__(self, kind="oracle", target="generic"):
        self.kind = kind
        self.target = target
        self.lib = oracle_lib() if kind == "oracle" else ref_lib(target)

    def fn(self, prec, name):
        if self.kind == "oracle":
            sym = "oracle_%s_%s" % (prec, name)
        else:
            # the compiled library spells the names the BLASFEO way
            bname = {"gemm_nt": "gemm_nt", "syrk_ln": "syrk_ln", "trsm_rltn": "trsm_rltn",
                     "potrf_l": "potrf_l", "syrk_potrf_ln": "syrk_%spotrf_ln" % prec,
                     "getrf_rp": "getrf_rp", "geqrf": "geqrf", "geqrf_worksize": "geqrf_worksize",
                     "trmm_rlnn": "trmm_rlnn", "trsv_lnn": "trsv_lnn", "trsv_ltn": "trsv_ltn",
                     "gemv_n": "gemv_n", "gecp": "gecp", "diare": "diare", "rowsw": "rowsw",
                     "syrk_ln_mn": "syrk_ln_mn", "trsm_rltu": "trsm_rltu", "potrf_l_mn": "potrf_l_mn",
                     "getrf_np": "getrf_np", "gemv_t": "gemv_t", "trmv_lnn": "trmv_lnn", "trmv_ltn": "trmv_ltn",
                     "trsv_lnn_mn": "trsv_lnn_mn", "trsv_ltn_mn": "trsv_ltn_mn"}[name]
            pre = "blasfeo_" if self.kind == "hp" else "blasfeo_ref_"
            sym = pre + prec + bname
        f = getattr(self.lib, sym)
        return f

    # ---- typed wrappers (prec = 'd' or 's') ----
    def _R(self, prec):
        return C.c_double if prec == "d" else C.c_float

    def gemm_nt(self, prec, m, n, k, alpha, A, ai, aj, B, bi, bj, beta, Cm, ci, cj, D, di, dj):
        R = self._R(prec)
        self.fn(prec, "gemm_nt")(m, n, k, R(alpha), A.ref, ai, aj, B.ref, bi, bj, R(beta), Cm.ref, ci, cj, D.ref, di, dj)

    def syrk_ln(self, prec, m, k, alpha, A, ai, aj, B, bi, bj, beta, Cm, ci, cj, D, di, dj):
        R = self._R(prec)
        self.fn(prec, "syrk_ln")(m, k, R(alpha), A.ref, ai, aj, B.ref, bi, bj, R(beta), Cm.ref, ci, cj, D.ref, di, dj)

    def trsm_rltn(self, prec, m, n, alpha, A, ai, aj, B, bi, bj, D, di, dj):
        R = self._R(prec)
        self.fn(prec, "trsm_rltn")(m, n, R(alpha), A.ref, ai, aj, B.ref, bi, bj, D.ref, di, dj)

    def potrf_l(self, prec, m, Cm, ci, cj, D, di, dj):
        self.fn(prec, "potrf_l")(m, Cm.ref, ci, cj, D.ref, di, dj)

    def syrk_potrf_ln(self, prec, m, k, A, ai, aj, B, bi, bj, Cm, ci, cj, D, di, dj):
        self.fn(prec, "syrk_potrf_ln")(m, k, A.ref, ai, aj, B.ref, bi, bj, Cm.ref, ci, cj, D.ref, di, dj)

    def getrf_rp(self, prec, m, n, Cm, ci, cj, D, di, dj):
        ipiv = np.zeros(max(1, min(m, n)) + 8, dtype=np.int32)
        self.fn(prec, "getrf_rp")(m, n, Cm.ref, ci, cj, D.ref, di, dj, ipiv.ctypes.data_as(C.POINTER(C.c_int)))
        return ipiv[: min(m, n)].copy()

    def geqrf(self, prec, m, n, Cm, ci, cj, D, di, dj):
        ws = self.fn(prec, "geqrf_worksize")
        ws.restype = C.c_int
        nbytes = max(int(ws(m, n)), 64)
        work = np.zeros(nbytes // 8 + 64, dtype=np.float64)
        # the HP kernels read aligned data from the work buffer
        addr = work.ctypes.data
        addr = (addr + 63) // 64 * 64
        self.fn(prec, "geqrf")(m, n, Cm.ref, ci, cj, D.ref, di, dj, C.c_void_p(addr))

    def syrk_ln_mn(self, prec, m, n, k, alpha, A, ai, aj, B, bi, bj, beta, Cm, ci, cj, D, di, dj):
        R = self._R(prec)
        self.fn(prec, "syrk_ln_mn")(m, n, k, R(alpha), A.ref, ai, aj, B.ref, bi, bj, R(beta), Cm.ref, ci, cj, D.ref,
                                    di, dj)

    def trsm_rltu(self, prec, m, n, alpha, A, ai, aj, B, bi, bj, D, di, dj):
        R = self._R(prec)
        self.fn(prec, "trsm_rltu")(m, n, R(alpha), A.ref, ai, aj, B.ref, bi, bj, D.ref, di, dj)

    def potrf_l_mn(self, prec, m, n, Cm, ci, cj, D, di, dj):
        self.fn(prec, "potrf_l_mn")(m, n, Cm.ref, ci, cj, D.ref, di, dj)

    def getrf_np(self, prec, m, n, Cm, ci, cj, D, di, dj):
        self.fn(prec, "getrf_np")(m, n, Cm.ref, ci, cj, D.ref, di, dj)

    def trmm_rlnn(self, prec, m, n, alpha, A, ai, aj, B, bi, bj, D, di, dj):
        R = self._R(prec)
        # reference argument order: (m, n, alpha, sB?, ...) is (m,n,alpha,sA,ai,aj,sB,bi,bj,sD,di,dj)
        self.fn(prec, "trmm_rlnn")(m, n, R(alpha), A.ref, ai, aj, B.ref, bi, bj, D.ref, di, dj)

    def trsv_lnn(self, prec, m, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trsv_lnn")(m, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def trsv_ltn(self, prec, m, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trsv_ltn")(m, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def gemv_t(self, prec, m, n, alpha, A, ai, aj, x, xi, beta, y, yi, z, zi):
        R = self._R(prec)
        self.fn(prec, "gemv_t")(m, n, R(alpha), A.ref, ai, aj, x.ref, xi, R(beta), y.ref, yi, z.ref, zi)

    def trmv_lnn(self, prec, m, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trmv_lnn")(m, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def trmv_ltn(self, prec, m, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trmv_ltn")(m, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def trsv_lnn_mn(self, prec, m, n, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trsv_lnn_mn")(m, n, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def trsv_ltn_mn(self, prec, m, n, A, ai, aj, x, xi, z, zi):
        self.fn(prec, "trsv_ltn_mn")(m, n, A.ref, ai, aj, x.ref, xi, z.ref, zi)

    def gemv_n(self, prec, m, n, alpha, A, ai, aj, x, xi, beta, y, yi, z, zi):
        R = self._R(prec)
        self.fn(prec, "gemv_n")(m, n, R(alpha), A.ref, ai, aj, x.ref, xi, R(beta), y.ref, yi, z.ref, zi)
