"""mdgpu_b200: B200-native multifrontal sparse Cholesky (Python front-end).

A thin ctypes layer over the C ABI in ``include/mdgpu_b200.h`` (library
``mdgpu_b200/libmdgpu_b200.so``).  The numeric phase runs only on the GPU:
when the library or a CUDA device is missing the calls raise instead of
falling back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdgpu_b200.so")

FP64, FP32, BF16, TF32 = 0, 1, 2, 3
ORDER_NATURAL, ORDER_AMD = 0, 1
TREE_NODAL, TREE_SUPER, TREE_RELAXED = 0, 1, 2

STATUS = {0: "ok", -1: "invalid argument", -2: "not positive definite", -3: "out of memory",
          -4: "CUDA error", -5: "elimination tree is a forest", -6: "invalid call order",
          -7: "no CUDA device"}

# every entry point declared in include/mdgpu_b200.h
EXPORTS = ("mdgpu_analyze", "mdgpu_analyze_batch", "mdgpu_analyze_tree", "mdgpu_destroy", "mdgpu_check_plan", "mdgpu_info",
           "mdgpu_estimate_batch", "mdgpu_get_array", "mdgpu_factor", "mdgpu_factor_device", "mdgpu_not_spd_column",
           "mdgpu_solve", "mdgpu_solve_device", "mdgpu_solve_device_noalloc", "mdgpu_refine",
           "mdgpu_refine_device", "mdgpu_gmres_ir", "mdgpu_gmres_ir_device",
           "mdgpu_get_L", "mdgpu_profile", "mdgpu_profile_read", "mdgpu_status_string",
           "mdgpu_last_error", "mdgpu_load_triplet", "mdgpu_logdet", "mdgpu_selinv",
           "mdgpu_grad_lower", "mdgpu_grad_lower_device", "mdgpu_adjoint",
           "mdgpu_adjoint_device", "mdgpu_autotune")

KERNEL_CLASSES = ("small_front", "assemble", "potrf", "panel", "schur_update", "solve_small",
                  "solve_large", "other")
# the roofline each class is measured against: the tensor pipes for the
# trailing (Schur) updates, HBM for the rest -- the diagonal-tile factor and
# the in-panel tile steps read and write 64 x 64 tiles, and their distance
# from streaming speed is the latency of the dependency chain
KERNEL_BOUND = {"small_front": "hbm", "assemble": "hbm", "potrf": "hbm", "panel": "hbm",
                "schur_update": "tensor", "solve_small": "hbm", "solve_large": "hbm",
                "other": "hbm"}


class MdgpuError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("%s (%d)%s" % (STATUS.get(status, "error"), status,
                                        (": " + msg) if msg else ""))


class NotSPDError(MdgpuError):
    def __init__(self, status, msg, column):
        super().__init__(status, msg)
        self.column = column


_lib = None


def lib():
    """Load the C-ABI library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libmdgpu_b200.so not built: run `make -C mdgpu_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_void_p, C.c_void_p
        L.mdgpu_analyze.argtypes = [C.c_int, ip, ip, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
        L.mdgpu_analyze_tree.argtypes = [C.c_int, ip, ip, C.c_int, ip, ip, ip, ip, ip,
                                         C.POINTER(vp)]
        L.mdgpu_analyze_batch.argtypes = [C.c_int, ip, C.POINTER(vp), C.POINTER(vp), C.c_int,
                                          C.c_int, C.c_int, C.POINTER(vp)]
        L.mdgpu_estimate_batch.argtypes = [C.c_int, ip, C.POINTER(vp), C.POINTER(vp), C.c_int,
                                           C.c_int, C.c_int, dp, vp]
        L.mdgpu_destroy.argtypes = [vp]
        L.mdgpu_check_plan.argtypes = [vp]
        L.mdgpu_destroy.restype = None
        L.mdgpu_info.argtypes = [vp, C.c_char_p, C.POINTER(C.c_longlong)]
        L.mdgpu_get_array.argtypes = [vp, C.c_char_p, vp]
        L.mdgpu_factor.argtypes = [vp, dp, C.c_int, vp]
        L.mdgpu_factor_device.argtypes = [vp, dp, C.c_int, vp]
        L.mdgpu_not_spd_column.argtypes = [vp]
        L.mdgpu_solve.argtypes = [vp, dp, C.c_int, dp, C.c_int, C.c_int, vp]
        L.mdgpu_solve_device.argtypes = [vp, dp, C.c_int, dp, C.c_int, C.c_int, vp]
        L.mdgpu_solve_device_noalloc.argtypes = [vp, dp, C.c_int, dp, C.c_int, C.c_int, vp]
        L.mdgpu_refine.argtypes = [vp, dp, C.c_int, dp, C.c_int, C.c_int, C.c_double, C.c_int,
                                   dp, vp, vp]
        L.mdgpu_refine_device.argtypes = L.mdgpu_refine.argtypes
        L.mdgpu_gmres_ir.argtypes = [vp, dp, C.c_int, dp, C.c_int, C.c_int, C.c_double, C.c_int,
                                     C.c_int, C.c_double, dp, vp, vp, vp]
        L.mdgpu_gmres_ir_device.argtypes = L.mdgpu_gmres_ir.argtypes
        L.mdgpu_get_L.argtypes = [vp, vp, vp, vp]
        L.mdgpu_profile.argtypes = [vp, C.c_int]
        L.mdgpu_profile_read.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.mdgpu_load_triplet.argtypes = [C.c_char_p, C.c_int, ip, ip, ip, vp, vp, vp]
        L.mdgpu_logdet.argtypes = [vp, vp, vp]
        L.mdgpu_selinv.argtypes = [vp, vp]
        L.mdgpu_grad_lower.argtypes = [vp, vp, vp, vp]
        L.mdgpu_grad_lower_device.argtypes = [vp, vp, vp, vp]
        L.mdgpu_adjoint.argtypes = [vp, vp, vp, vp]
        L.mdgpu_adjoint_device.argtypes = [vp, vp, vp, vp]
        L.mdgpu_autotune.argtypes = [vp, vp, C.c_int, vp]
        L.mdgpu_status_string.argtypes = [C.c_int]
        L.mdgpu_status_string.restype = C.c_char_p
        L.mdgpu_last_error.restype = C.c_char_p
        for name in EXPORTS:
            f = getattr(L, name)
            if f.restype is C.c_int and name not in ("mdgpu_not_spd_column",):
                pass
        _lib = L
    return _lib


def _check(rc, h=None):
    if rc == 0:
        return
    msg = lib().mdgpu_last_error().decode()
    if rc == -2 and h is not None:
        raise NotSPDError(rc, msg, lib().mdgpu_not_spd_column(h))
    raise MdgpuError(rc, msg)


def _ptr(a):
    return a.ctypes.data


def _tensor_ptr(t):
    return C.c_void_p(t.data_ptr())


def _dev_stream(stream):
    """The stream for a call on CUDA tensors: the caller's, else torch's
    current stream, so the call is ordered with the torch work that made its
    inputs and with the torch work that reads its outputs."""
    if stream is not None:
        return stream
    import torch

    s = torch.cuda.current_stream().cuda_stream
    # torch's default stream is the legacy NULL stream (handle 0), which the
    # library would read as "no stream given": name it cudaStreamLegacy (1)
    return C.c_void_p(s if s else 1)


def load_triplet(path, matrix_market=False):
    """Read a matrix file as the reference's cs_load + cs_compress do
    (1-based "i j x" triples until the first line that is not one), or a
    Matrix Market real coordinate file.  Returns (m, n, Ap, Ai, Ax): int32
    column pointers and 0-based rows, float64 values, a column's entries in
    file order."""
    L = lib()
    m, n, nnz = C.c_int(), C.c_int(), C.c_int()
    fmt = 1 if matrix_market else 0
    p = str(path).encode()
    _check(L.mdgpu_load_triplet(p, fmt, C.byref(m), C.byref(n), C.byref(nnz), None, None, None))
    Ap = np.zeros(n.value + 1, np.int32)
    Ai = np.zeros(max(nnz.value, 1), np.int32)
    Ax = np.zeros(max(nnz.value, 1), np.float64)
    _check(L.mdgpu_load_triplet(p, fmt, C.byref(m), C.byref(n), C.byref(nnz), _ptr(Ap), _ptr(Ai),
                                _ptr(Ax)))
    return m.value, n.value, Ap, Ai[: nnz.value], Ax[: nnz.value]


def estimate_batch(systems, ordering=ORDER_AMD, tree=TREE_SUPER, relax_zeros=0):
    """Flop count and L entries of each of the independent systems
    [(n, Ap, Ai), ...] from their symbolic analyses (host only, all cores);
    returns (flops, lnz) arrays."""
    ns = len(systems)
    nn = np.array([int(s[0]) for s in systems], dtype=np.int32)
    Aps = [np.ascontiguousarray(s[1], dtype=np.int32) for s in systems]
    Ais = [np.ascontiguousarray(s[2], dtype=np.int32) for s in systems]
    pa = (C.c_void_p * ns)(*[a.ctypes.data for a in Aps])
    pi = (C.c_void_p * ns)(*[a.ctypes.data for a in Ais])
    flops = np.zeros(ns)
    lnz = np.zeros(ns, np.int64)
    _check(lib().mdgpu_estimate_batch(ns, _ptr(nn), pa, pi, int(ordering), int(tree),
                                      int(relax_zeros), _ptr(flops), _ptr(lnz)))
    return flops, lnz


class Solver:
    """One sparsity pattern: symbolic analysis at construction, then any
    number of GPU factorizations and solves.

    ``Ap, Ai`` describe the lower triangle (diagonal included) in compressed
    columns with sorted rows, int32 -- the reference's ``cs`` layout.
    """

    def __init__(self, n, Ap, Ai, ordering=ORDER_AMD, tree=TREE_SUPER, relax_zeros=0):
        L = lib()
        self.n = int(n)
        self.Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        self.Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        self._h = C.c_void_p()
        _check(L.mdgpu_analyze(self.n, _ptr(self.Ap), _ptr(self.Ai), int(ordering), int(tree),
                               int(relax_zeros), C.byref(self._h)))

    @classmethod
    def batch(cls, systems, ordering=ORDER_AMD, tree=TREE_SUPER, relax_zeros=0):
        """Many independent systems [(n, Ap, Ai), ...] under one solver: each
        analysed on its own, numbered one after another (block-diagonal).
        Values and right-hand sides are the systems' arrays concatenated;
        ``row_off`` / ``val_off`` give each system's slice."""
        self = cls.__new__(cls)
        L = lib()
        ns = len(systems)
        nn = np.array([int(s[0]) for s in systems], dtype=np.int32)
        Aps = [np.ascontiguousarray(s[1], dtype=np.int32) for s in systems]
        Ais = [np.ascontiguousarray(s[2], dtype=np.int32) for s in systems]
        self._keep = (nn, Aps, Ais)
        pa = (C.c_void_p * ns)(*[a.ctypes.data for a in Aps])
        pi = (C.c_void_p * ns)(*[a.ctypes.data for a in Ais])
        self._h = C.c_void_p()
        _check(L.mdgpu_analyze_batch(ns, _ptr(nn), pa, pi, int(ordering), int(tree),
                                     int(relax_zeros), C.byref(self._h)))
        self.n = int(nn.sum())
        self.Ap = None
        self.Ai = None
        self.row_off = self.array("sys_row_off")
        self.val_off = self.array("sys_val_off")
        return self

    @classmethod
    def from_tree(cls, n, Ap, Ai, first_col, ncols, child_ptr, child, count):
        self = cls.__new__(cls)
        L = lib()
        self.n = int(n)
        self.Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        self.Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        arrs = [np.ascontiguousarray(a, dtype=np.int32)
                for a in (first_col, ncols, child_ptr, child, count)]
        self._keep = arrs
        self._h = C.c_void_p()
        _check(L.mdgpu_analyze_tree(self.n, _ptr(self.Ap), _ptr(self.Ai), len(arrs[0]),
                                    *[_ptr(a) for a in arrs], C.byref(self._h)))
        return self

    def close(self):
        if getattr(self, "_h", None):
            lib().mdgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check_plan(self):
        """Host check of every invariant of the plan's tables (raises
        MdgpuError naming the failed invariant)."""
        _check(lib().mdgpu_check_plan(self._h))

    def info(self, key):
        v = C.c_longlong()
        _check(lib().mdgpu_info(self._h, key.encode(), C.byref(v)))
        return v.value

    def array(self, name):
        n, ns = self.n, self.info("nsuper")
        sizes = {"perm": n, "parent": n, "post": n, "count0": n, "count": n, "relax_perm": n,
                 "sn_first": ns, "sn_ncols": ns, "child_ptr": ns + 1,
                 "child": self.info("nchild"), "rows_ptr": ns + 1,
                 "rows": self.info("rows_total"), "relmap": self.info("rows_total"),
                 "level": ns, "sys_row_off": self.info("nsys") + 1,
                 "sys_val_off": self.info("nsys") + 1,
                 "warp_list": self.info("small_fronts"), "warp_cnt": 3 * self.info("nlevels"),
                 "amap_off": ns, "amap_row": self.info("amap_rows"),
                 "amap_ent": self.info("amap_entries")}
        if name == "Lp":
            a = np.zeros(n + 1, np.int64)
        else:
            a = np.zeros(max(sizes[name], 1), np.int32)
        _check(lib().mdgpu_get_array(self._h, name.encode(), _ptr(a)))
        return a if name == "Lp" else a[: sizes[name]]

    # ---- numeric -----------------------------------------------------
    def factor(self, Ax, precision=FP64, stream=None):
        """Ax: numpy float64 (host) or a CUDA torch tensor (device).  Every
        successful factor advances self.generation (which factor the handle
        holds: callers that keep results across factors compare it)."""
        if hasattr(Ax, "data_ptr"):
            _check(lib().mdgpu_factor_device(self._h, _tensor_ptr(Ax), int(precision),
                                             _dev_stream(stream)),
                   self._h)
        else:
            Ax = np.ascontiguousarray(Ax, dtype=np.float64)
            _check(lib().mdgpu_factor(self._h, _ptr(Ax), int(precision), stream), self._h)
        self.generation = getattr(self, "generation", 0) + 1

    def _device_layout(self, T):
        """(nrhs, leading dimension) of a column-major float64 CUDA tensor of
        shape (n,) or (n, k); raises on any other layout."""
        import torch

        if T.dtype != torch.float64 or not T.is_cuda:
            raise ValueError("device vectors must be float64 CUDA tensors")
        if T.dim() == 1:
            if T.shape[0] != self.n or (self.n > 1 and T.stride(0) != 1):
                raise ValueError("device vector must be contiguous of length n")
            return 1, self.n
        if T.dim() != 2 or T.shape[0] != self.n:
            raise ValueError("device right-hand sides must have shape (n, k)")
        if self.n > 1 and T.stride(0) != 1:
            raise ValueError("device right-hand sides must be column-major (B.T.contiguous().T)")
        # a single column's stride is arbitrary in torch (size-1 dimension)
        return T.shape[1], (self.n if T.shape[1] == 1 else T.stride(1))

    def solve(self, B, stream=None):
        """B: (n,) or (n, k) float64 numpy array, or CUDA torch tensors.
        Device tensors must be column-major contiguous (use B.T.contiguous().T)."""
        if hasattr(B, "data_ptr"):
            import torch

            nrhs, ld = self._device_layout(B)
            X = torch.empty((nrhs, self.n), dtype=B.dtype, device=B.device).t()
            _check(lib().mdgpu_solve_device(self._h, _tensor_ptr(B), ld, _tensor_ptr(X),
                                            self.n, nrhs, _dev_stream(stream)))
            return X[:, 0] if B.dim() == 1 else X
        B = np.asarray(B, dtype=np.float64)
        one = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(self.n, -1))
        X = np.zeros_like(Bf, order="F")
        _check(lib().mdgpu_solve(self._h, _ptr(Bf), self.n, _ptr(X), self.n, Bf.shape[1],
                                 stream))
        return X[:, 0] if one else X

    def refine(self, B, tol=1e-14, maxit=10, stream=None):
        """Solve with FP64 iterative refinement; returns (x, berr, iters)."""
        B = np.asarray(B, dtype=np.float64)
        one = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(self.n, -1))
        X = np.zeros_like(Bf, order="F")
        berr = np.zeros(Bf.shape[1])
        it = C.c_int()
        _check(lib().mdgpu_refine(self._h, _ptr(Bf), self.n, _ptr(X), self.n, Bf.shape[1],
                                  float(tol), int(maxit), _ptr(berr), C.byref(it), stream))
        return (X[:, 0] if one else X), berr, it.value

    def refine_device(self, B, X, tol=1e-14, maxit=10, stream=None):
        nrhs, ldb = self._device_layout(B)
        nx, ldx = self._device_layout(X)
        if nx != nrhs:
            raise ValueError("B and X hold different numbers of right-hand sides")
        berr = np.zeros(nrhs)
        it = C.c_int()
        _check(lib().mdgpu_refine_device(self._h, _tensor_ptr(B), ldb, _tensor_ptr(X), ldx, nrhs,
                                         float(tol), int(maxit), _ptr(berr), C.byref(it),
                                         _dev_stream(stream)))
        return berr, it.value

    def gmres_ir(self, B, tol=1e-14, maxit=10, restart=30, inner_tol=1e-8, stream=None):
        """Solve with GMRES-based iterative refinement (the factor's solve as
        the preconditioner of GMRES in FP64); returns (x, berr, iters, inner)
        with one backward error, correction count and GMRES step count per
        right-hand side."""
        B = np.asarray(B, dtype=np.float64)
        one = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(self.n, -1))
        X = np.zeros_like(Bf, order="F")
        k = Bf.shape[1]
        berr = np.zeros(k)
        it = np.zeros(k, np.int32)
        inner = np.zeros(k, np.int32)
        _check(lib().mdgpu_gmres_ir(self._h, _ptr(Bf), self.n, _ptr(X), self.n, k, float(tol),
                                    int(maxit), int(restart), float(inner_tol), _ptr(berr),
                                    _ptr(it), _ptr(inner), stream))
        if one:
            return X[:, 0], berr[0], int(it[0]), int(inner[0])
        return X, berr, it, inner

    def gmres_ir_device(self, B, X, tol=1e-14, maxit=10, restart=30, inner_tol=1e-8,
                        stream=None):
        """GMRES-IR on CUDA tensors (column-major); returns (berr, iters, inner)."""
        nrhs, ldb = self._device_layout(B)
        nx, ldx = self._device_layout(X)
        if nx != nrhs:
            raise ValueError("B and X hold different numbers of right-hand sides")
        berr = np.zeros(nrhs)
        it = np.zeros(nrhs, np.int32)
        inner = np.zeros(nrhs, np.int32)
        _check(lib().mdgpu_gmres_ir_device(self._h, _tensor_ptr(B), ldb, _tensor_ptr(X), ldx,
                                           nrhs, float(tol), int(maxit), int(restart),
                                           float(inner_tol), _ptr(berr), _ptr(it), _ptr(inner),
                                           _dev_stream(stream)))
        return berr, it, inner

    def profile_step(self, fn):
        """Run fn() once with per-launch event timing on; return per-class
        totals and the dominant class (most device time)."""
        _check(lib().mdgpu_profile(self._h, 1))
        fn()
        _check(lib().mdgpu_profile(self._h, 0))
        classes = {}
        total_launches = 0
        for k, name in enumerate(KERNEL_CLASSES):
            ms, n, fl, by = C.c_double(), C.c_longlong(), C.c_double(), C.c_double()
            _check(lib().mdgpu_profile_read(self._h, k, C.byref(ms), C.byref(n), C.byref(fl),
                                            C.byref(by)))
            if n.value:
                classes[name] = {"ms": ms.value, "launches": n.value, "flops": fl.value,
                                 "bytes": by.value, "bound": KERNEL_BOUND[name]}
                total_launches += n.value
        dom = max(classes, key=lambda k: classes[k]["ms"]) if classes else None
        return {"classes": classes, "dominant": dom, "launches_per_step": total_launches}

    # ---- differentiation ----------------------------------------------
    def logdet(self, stream=None):
        """log det A from the current factor."""
        v = C.c_double()
        _check(lib().mdgpu_logdet(self._h, C.byref(v), stream), self._h)
        return v.value

    def selinv(self, stream=None):
        """Selected inverse of the current FP64 factor (kept on the device)."""
        _check(lib().mdgpu_selinv(self._h, stream), self._h)

    def grad_lower(self, x=None, stream=None):
        """d(log det A + b' A^-1 b) / d Ax for the caller's lower-triangle
        values, x = A^-1 b (None: the gradient of log det A alone); numpy x
        gives a numpy G, a CUDA tensor x (or x None with device=True) a CUDA
        tensor."""
        nnz = self.info("nnz")
        if x is not None and hasattr(x, "data_ptr"):
            import torch

            G = torch.empty(nnz, dtype=torch.float64, device=x.device)
            _check(lib().mdgpu_grad_lower_device(self._h, _tensor_ptr(x), _tensor_ptr(G),
                                                 _dev_stream(stream)), self._h)
            return G
        G = np.zeros(max(nnz, 1))
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        _check(lib().mdgpu_grad_lower(self._h, None if xa is None else _ptr(xa), _ptr(G), stream),
               self._h)
        return G[:nnz]

    def autotune(self, Ax, precision=FP64):
        """Choose the small-front kernels' launch shapes for this handle by
        timing the factor of Ax (numpy); returns the chosen shapes and the
        factor time in ms."""
        Ax = np.ascontiguousarray(Ax, dtype=np.float64)
        ms = C.c_double()
        _check(lib().mdgpu_autotune(self._h, _ptr(Ax), int(precision), C.byref(ms)), self._h)
        out = {"tiny_blocks": self.info("tune_tiny_blocks"), "ms": ms.value}
        for b in range(2, 6):
            out["threads_b%d" % b] = self.info("tune_threads_b%d" % b)
        return out

    def adjoint(self, Lbar, stream=None):
        """Reverse mode of the current FP64 factorization: Lbar, the gradient
        of a loss with respect to L's values (lnz entries, get_L's order) ->
        the gradient with respect to the caller's lower-triangle values (nnz
        entries, caller order).  numpy in, numpy out; a CUDA tensor in, a
        CUDA tensor out."""
        nnz = self.info("nnz")
        if hasattr(Lbar, "data_ptr"):
            import torch

            G = torch.empty(max(nnz, 1), dtype=torch.float64, device=Lbar.device)
            Lc = Lbar.contiguous()
            _check(lib().mdgpu_adjoint_device(self._h, _tensor_ptr(Lc), _tensor_ptr(G),
                                              _dev_stream(stream)), self._h)
            return G[:nnz]
        Lb = np.ascontiguousarray(Lbar, dtype=np.float64)
        G = np.zeros(max(nnz, 1))
        _check(lib().mdgpu_adjoint(self._h, _ptr(Lb), _ptr(G), stream), self._h)
        return G[:nnz]

    def get_L(self, values=True):
        """L as (Lp int64, Li int32, Lx float64) -- the reference's spL."""
        lnz = self.info("lnz")
        Lp = np.zeros(self.n + 1, np.int64)
        Li = np.zeros(max(lnz, 1), np.int32)
        Lx = np.zeros(max(lnz, 1), np.float64) if values else None
        _check(lib().mdgpu_get_L(self._h, _ptr(Lp), _ptr(Li),
                                 _ptr(Lx) if values else None))
        return Lp, Li[:lnz], (Lx[:lnz] if values else None)
