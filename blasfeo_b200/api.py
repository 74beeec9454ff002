"""Python mirror of the BLASFEO API over libblasfeo_b200.so.

Routines keep the reference names and argument order; matrices are
:class:`DMat` / :class:`SMat` objects whose storage is device memory.  Example::

    A = DMat(64, 64).pack(a_host)          # blasfeo_create_dmat + blasfeo_pack_dmat
    D = DMat(64, 64)
    blasfeo_dpotrf_l(64, A, 0, 0, D, 0, 0)
    L = D.unpack()

Device buffers are torch CUDA tensors (allocation only); every computation
runs in the CUDA kernels of the shared library.
"""
import ctypes as C

import numpy as np

from . import lib, dmat, smat, dvec, svec, dmat_batch, smat_batch, dmat_batch_il, cm_dmat, cm_smat, check

__all__ = [
    "DMat", "SMat", "DVec", "SVec", "DMatBatch", "SMatBatch", "DMatBatchIL", "device_buffer", "set_stream", "set_sync",
    "set_posv_engine", "POSV_DEFAULT", "POSV_SIMT", "POSV_TENSOR",
    "blasfeo_dgemm_nt", "blasfeo_dsyrk_ln", "blasfeo_dtrsm_rltn", "blasfeo_dtrmm_rlnn", "blasfeo_dpotrf_l",
    "blasfeo_dsyrk_dpotrf_ln", "blasfeo_dgetrf_rp", "blasfeo_dgeqrf", "blasfeo_dgeqrf_worksize",
    "blasfeo_sgemm_nt", "blasfeo_ssyrk_ln", "blasfeo_strsm_rltn", "blasfeo_strmm_rlnn", "blasfeo_spotrf_l",
    "blasfeo_ssyrk_spotrf_ln", "blasfeo_sgetrf_rp", "blasfeo_sgeqrf", "blasfeo_sgeqrf_worksize",
    "blasfeo_dgecp", "blasfeo_ddiare", "blasfeo_drowsw", "blasfeo_dgemv_n", "blasfeo_dtrsv_lnn",
    "blasfeo_dtrsv_ltn", "descriptor_array", "vector_array",
    "blasfeo_dsyrk_ln_mn", "blasfeo_dtrsm_rltu", "blasfeo_dpotrf_l_mn", "blasfeo_dgetrf_np",
    "blasfeo_ssyrk_ln_mn", "blasfeo_strsm_rltu", "blasfeo_spotrf_l_mn", "blasfeo_sgetrf_np",
    "CmDMat", "CmSMat", "blasfeo_cm_dgemm_nt", "blasfeo_cm_dsyrk_ln", "blasfeo_cm_dtrsm_rltn",
    "blasfeo_cm_dpotrf_l", "blasfeo_cm_dgetrf_rp", "blasfeo_cm_sgemm_nt", "blasfeo_cm_strsm_rltn",
    "blasfeo_cm_spotrf_l",
]


def device_buffer(nbytes):
    """A zero-filled device allocation of at least nbytes (torch uint8 tensor)."""
    import torch
    return torch.zeros(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def set_stream(stream):
    """Stream of the single-instance calls (a torch.cuda.Stream, an int handle or None)."""
    h = getattr(stream, "cuda_stream", stream)
    lib.blasfeo_b200_set_stream(C.c_void_p(h or 0))


def set_sync(sync):
    lib.blasfeo_b200_set_sync(1 if sync else 0)


POSV_DEFAULT, POSV_SIMT, POSV_TENSOR = 0, 1, 2


def set_posv_engine(engine):
    """Engine of blasfeo_dsposv_l_vbatch for n <= 256 (this host thread):
    POSV_SIMT, POSV_TENSOR or POSV_DEFAULT; returns the previous engine."""
    prev = lib.blasfeo_b200_get_posv_engine()
    check(lib.blasfeo_b200_set_posv_engine(int(engine)))
    return prev


class _Mat:
    _prec = "d"
    _np = np.float64
    _desc = dmat

    def __init__(self, m, n, buffer=None, offset=0):
        self.m, self.n = m, n
        nbytes = getattr(lib, "blasfeo_memsize_%smat" % self._prec)(m, n)
        if buffer is None:
            buffer = device_buffer(nbytes)
            offset = 0
        self.buf = buffer
        self.s = self._desc()
        getattr(lib, "blasfeo_create_%smat" % self._prec)(m, n, C.byref(self.s), C.c_void_p(buffer.data_ptr() + offset))

    @property
    def ref(self):
        return C.byref(self.s)

    def pack(self, A, ai=0, aj=0):
        A = np.asfortranarray(np.asarray(A, dtype=self._np))
        m, n = A.shape
        getattr(lib, "blasfeo_pack_%smat" % self._prec)(m, n, A.ctypes.data, m, self.ref, ai, aj)
        check()
        return self

    def unpack(self, m=None, n=None, ai=0, aj=0):
        m = self.m - ai if m is None else m
        n = self.n - aj if n is None else n
        out = np.zeros((m, n), dtype=self._np, order="F")
        getattr(lib, "blasfeo_unpack_%smat" % self._prec)(m, n, self.ref, ai, aj, out.ctypes.data, m)
        check()
        return np.ascontiguousarray(out)

    def diag_array(self, k=None):
        """The dA array (inverse diagonal / tau) copied to the host."""
        import torch
        k = min(self.m, self.n) if k is None else k
        esz = np.dtype(self._np).itemsize
        off = self.s.dA - self.buf.data_ptr()
        t = self.buf[off:off + k * esz].cpu().numpy().view(self._np)
        return t.copy()

    @property
    def use_dA(self):
        return self.s.use_dA


class DMat(_Mat):
    pass


class SMat(_Mat):
    _prec = "s"
    _np = np.float32
    _desc = smat


class _Vec:
    _prec = "d"
    _np = np.float64
    _desc = dvec

    def __init__(self, m, buffer=None, offset=0):
        self.m = m
        nbytes = getattr(lib, "blasfeo_memsize_%svec" % self._prec)(m)
        if buffer is None:
            buffer = device_buffer(nbytes)
            offset = 0
        self.buf = buffer
        self.s = self._desc()
        getattr(lib, "blasfeo_create_%svec" % self._prec)(m, C.byref(self.s), C.c_void_p(buffer.data_ptr() + offset))

    @property
    def ref(self):
        return C.byref(self.s)

    def pack(self, x, ai=0):
        x = np.ascontiguousarray(np.asarray(x, dtype=self._np))
        getattr(lib, "blasfeo_pack_%svec" % self._prec)(len(x), x.ctypes.data, 0, self.ref, ai)
        check()
        return self

    def unpack(self, m=None, ai=0):
        m = self.m - ai if m is None else m
        out = np.zeros(m, dtype=self._np)
        getattr(lib, "blasfeo_unpack_%svec" % self._prec)(m, self.ref, ai, out.ctypes.data, 0)
        check()
        return out


class DVec(_Vec):
    pass


class SVec(_Vec):
    _prec = "s"
    _np = np.float32
    _desc = svec


class _MatBatch:
    """A uniform batch slab (struct blasfeo_dmat_batch)."""
    _prec = "d"
    _np = np.float64
    _desc = dmat_batch
    _inst = DMat

    def __init__(self, m, n, batch):
        self.m, self.n, self.batch = m, n, batch
        nbytes = getattr(lib, "blasfeo_memsize_%smat_batch" % self._prec)(m, n, batch)
        self.buf = device_buffer(nbytes)
        self.s = self._desc()
        getattr(lib, "blasfeo_create_%smat_batch" % self._prec)(m, n, batch, C.byref(self.s),
                                                                 C.c_void_p(self.buf.data_ptr()))

    @property
    def ref(self):
        return C.byref(self.s)

    @property
    def per_bytes(self):
        return self.s.stride * np.dtype(self._np).itemsize

    def pack_all(self, arr):
        """arr: (batch, m, n) host array -> device slab (panel-major per instance), one copy."""
        import torch
        arr = np.asarray(arr, dtype=self._np)
        b, m, n = arr.shape
        pm, cn = self.s.pm, self.s.cn
        host = np.zeros((b, self.s.stride), dtype=self._np)
        pad = np.zeros((b, pm, cn), dtype=self._np)
        pad[:, :m, :n] = arr
        # panel-major: [panel][col][row in panel]
        pan = pad.reshape(b, pm // 4, 4, cn).transpose(0, 1, 3, 2).reshape(b, pm * cn)
        host[:, : pm * cn] = pan
        t = torch.from_numpy(host.view(np.uint8).reshape(-1))
        self.buf[: t.numel()].copy_(t.to(self.buf.device))
        return self

    def unpack_all(self, m=None, n=None):
        m = self.m if m is None else m
        n = self.n if n is None else n
        pm, cn = self.s.pm, self.s.cn
        raw = self.buf[: self.batch * self.per_bytes].cpu().numpy().view(self._np).reshape(self.batch, self.s.stride)
        pan = raw[:, : pm * cn].reshape(self.batch, pm // 4, cn, 4).transpose(0, 1, 3, 2).reshape(self.batch, pm, cn)
        return np.ascontiguousarray(pan[:, :m, :n])

    def diag_all(self, k=None):
        k = min(self.m, self.n) if k is None else k
        pm, cn = self.s.pm, self.s.cn
        raw = self.buf[: self.batch * self.per_bytes].cpu().numpy().view(self._np).reshape(self.batch, self.s.stride)
        return raw[:, pm * cn: pm * cn + k].copy()


class DMatBatch(_MatBatch):
    pass


class SMatBatch(_MatBatch):
    _prec = "s"
    _np = np.float32
    _desc = smat_batch
    _inst = SMat


class DMatBatchIL:
    """A batch-interleaved slab (struct blasfeo_dmat_batch_il): element slot e
    of instance b at mem[(b // 16) * gstride + 16 e + b % 16]."""

    def __init__(self, m, n, batch):
        self.m, self.n, self.batch = m, n, batch
        nbytes = lib.blasfeo_memsize_dmat_batch_il(m, n, batch)
        self.buf = device_buffer(nbytes)
        self.s = dmat_batch_il()
        lib.blasfeo_create_dmat_batch_il(m, n, batch, C.byref(self.s), C.c_void_p(self.buf.data_ptr()))

    @property
    def ref(self):
        return C.byref(self.s)

    def from_batch(self, B, stream=None):
        check(lib.blasfeo_dmat_batch_to_il(B.ref, self.ref, stream))
        return self

    def to_batch(self, B, stream=None):
        check(lib.blasfeo_dmat_batch_from_il(self.ref, B.ref, stream))
        return B

    def pack_all(self, arr, stream=None):
        """arr: (batch, m, n) host array -> the slab, through
        blasfeo_pack_dmat_batch_il (host column-major, one host copy)."""
        arr = np.asarray(arr, dtype=np.float64)
        b, m, n = arr.shape
        cm = np.ascontiguousarray(arr.transpose(0, 2, 1))  # column-major per instance, lda = m
        check(lib.blasfeo_pack_dmat_batch_il(b, m, n, cm.ctypes.data_as(C.c_void_p), m, m * n, self.ref, stream))
        return self

    def unpack_all(self, m=None, n=None, stream=None):
        m = self.m if m is None else m
        n = self.n if n is None else n
        cm = np.zeros((self.batch, n, m), dtype=np.float64)
        check(lib.blasfeo_unpack_dmat_batch_il(self.batch, m, n, self.ref, cm.ctypes.data_as(C.c_void_p), m, m * n,
                                               stream))
        return np.ascontiguousarray(cm.transpose(0, 2, 1))


def descriptor_array(mats):
    """Device array of struct blasfeo_dmat descriptors (for the *_vbatch calls)."""
    import torch
    raw = b"".join(bytes(m.s) for m in mats)
    t = torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()
    return t


def vector_array(vecs):
    import torch
    raw = b"".join(bytes(v.s) for v in vecs)
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()


class _CmMat:
    """A column-major device matrix (struct blasfeo_cm_dmat): m x n, leading
    dimension m, created by blasfeo_cm_create_dmat on a device buffer."""
    _prec = "d"
    _np = np.float64
    _desc = cm_dmat

    def __init__(self, m, n):
        self.m, self.n = m, n
        nbytes = getattr(lib, "blasfeo_cm_memsize_%smat" % self._prec)(m, n)
        self.buf = device_buffer(nbytes)
        self.s = self._desc()
        getattr(lib, "blasfeo_cm_create_%smat" % self._prec)(m, n, C.byref(self.s), C.c_void_p(self.buf.data_ptr()))

    @property
    def ref(self):
        return C.byref(self.s)

    def _view(self):
        import torch
        esz = np.dtype(self._np).itemsize
        t = self.buf[: self.m * self.n * esz].view(torch.float64 if self._prec == "d" else torch.float32)
        return t.view(self.n, self.m)  # row j of the view = column j of the matrix

    def pack(self, A):
        import torch
        A = np.asarray(A, dtype=self._np)
        assert A.shape == (self.m, self.n)
        self._view().copy_(torch.from_numpy(np.ascontiguousarray(A.T)))
        return self

    def unpack(self):
        return np.ascontiguousarray(self._view().cpu().numpy().T)


class CmDMat(_CmMat):
    pass


class CmSMat(_CmMat):
    _prec = "s"
    _np = np.float32
    _desc = cm_smat


def _wrap(name):
    f = getattr(lib, name)

    def call(*args):
        conv = [a.ref if isinstance(a, (_Mat, _Vec, _CmMat)) else a for a in args]
        r = f(*conv)
        check()
        return r
    call.__name__ = name
    return call


for _p in ("d", "s"):
    for _r in ("gemm_nt", "syrk_ln", "trsm_rltn", "trmm_rlnn", "potrf_l", "geqrf_worksize", "gecp", "diare",
               "rowsw", "syrk_ln_mn", "trsm_rltu", "potrf_l_mn", "getrf_np"):
        globals()["blasfeo_%s%s" % (_p, _r)] = _wrap("blasfeo_%s%s" % (_p, _r))
    globals()["blasfeo_%ssyrk_%spotrf_ln" % (_p, _p)] = _wrap("blasfeo_%ssyrk_%spotrf_ln" % (_p, _p))
for _r in ("dgemv_n", "dtrsv_lnn", "dtrsv_ltn", "cm_dgemm_nt", "cm_dsyrk_ln", "cm_dtrsm_rltn", "cm_dpotrf_l",
           "cm_sgemm_nt", "cm_strsm_rltn", "cm_spotrf_l"):
    globals()["blasfeo_" + _r] = _wrap("blasfeo_" + _r)


def _getrf(prec, cm=False):
    f = getattr(lib, "blasfeo_%s%sgetrf_rp" % ("cm_" if cm else "", prec))

    def call(m, n, sC, ci, cj, sD, di, dj, ipiv=None):
        mn = max(1, min(m, n))
        buf = (C.c_int * mn)()
        f(m, n, sC.ref, ci, cj, sD.ref, di, dj, buf)
        check()
        piv = np.frombuffer(buf, dtype=np.int32, count=min(m, n)).copy()
        if ipiv is not None:
            ipiv[: len(piv)] = piv
        return piv
    return call


def _geqrf(prec):
    f = getattr(lib, "blasfeo_%sgeqrf" % prec)

    def call(m, n, sC, ci, cj, sD, di, dj, work=None):
        f(m, n, sC.ref, ci, cj, sD.ref, di, dj, None)
        check()
    return call


blasfeo_dgetrf_rp = _getrf("d")
blasfeo_sgetrf_rp = _getrf("s")
blasfeo_cm_dgetrf_rp = _getrf("d", cm=True)
blasfeo_dgeqrf = _geqrf("d")
blasfeo_sgeqrf = _geqrf("s")
