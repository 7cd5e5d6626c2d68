"""Python binding of libfmmg.so (include/fmmg.h): the B200 KIFMM3d evaluator.

``FMM3d`` mirrors the reference ``FMM3d_MPI`` object (fmm3d_mpi/fmm3d_mpi.hpp:36-249):
set ``knl``/``np``/``ctr``/``root_level`` through the constructor, call
``setup(src, nrm, trg)`` once per geometry, then ``evaluate(src_den)`` as often
as needed, and ``check()`` for the sampled dense-sum error of the reference
check() (fmm3d_mpi/fmm3d_check_mpi.cpp:34-172).  Device tensors (torch) go
through ``evaluate_device``.

The library is the only compute path: if libfmmg.so is missing or cannot load,
every call raises; nothing falls back to a CPU implementation.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmmg.so")

FMMG_OK, FMMG_INVALID_ARG, FMMG_OOM, FMMG_CUDA_ERROR, FMMG_TIMEOUT, FMMG_NOT_SUPPORTED, FMMG_STATE = range(7)
PREC_FP64, PREC_MIXED = 0, 1
STAGE_UP, STAGE_U, STAGE_V, STAGE_W, STAGE_X, STAGE_DOWN = 1, 2, 4, 8, 16, 32
STAGE_ALL = 63
STAGE_NAMES = ("upward", "ulist", "vlist", "wlist", "xlist", "downward", "total")
KERNEL_NAMES = ("prep", "s2m", "up_gemm", "p2p_near", "m2l_fwd", "m2l_had", "m2l_inv", "m2t", "s2l", "dn_gemm",
                "l2t", "scatter")

# kernel ids accepted by setup() (fmm3d_mpi/fmm3d_setup_mpi.cpp:113-126)
KERNELS = {111: (1, 1), 121: (1, 1), 311: (3, 3), 312: (3, 1), 321: (3, 3), 322: (3, 1), 511: (3, 3),
           521: (3, 3)}


class FmmgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("fmmg status %d: %s" % (status, msg))
        self.status = status


class _Options(ctypes.Structure):
    _fields_ = [("kernel_type", ctypes.c_int), ("coefs", ctypes.c_double * 2), ("np", ctypes.c_int),
                ("pts_max", ctypes.c_int), ("max_level", ctypes.c_int), ("ctr", ctypes.c_double * 3),
                ("root_level", ctypes.c_int), ("device", ctypes.c_int), ("stream", ctypes.c_void_p)]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile libfmmg.so in-tree (nvcc, sm_100a)."""
    subprocess.check_call(["make", "-s", "-j8", "-C", _HERE])


# every symbol include/fmmg.h declares, with its ctypes signature
SIGNATURES = {
    "fmmg_default_options": ([ctypes.POINTER(_Options)], ctypes.c_int),
    "fmmg_create": ([ctypes.POINTER(_Options), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "fmmg_setup": ([ctypes.c_void_p, ctypes.c_int64, _dp, _dp, ctypes.c_int64, _dp], ctypes.c_int),
    "fmmg_evaluate": ([ctypes.c_void_p, _dp, _dp], ctypes.c_int),
    "fmmg_evaluate_host": ([ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int], ctypes.c_int),
    "fmmg_evaluate_device": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
                             ctypes.c_int),
    "fmmg_synchronize": ([ctypes.c_void_p], ctypes.c_int),
    "fmmg_adjoint_device": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p], ctypes.c_int),
    "fmmg_adjoint_host": ([ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp], ctypes.c_int),
    "fmmg_evaluate_stages": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
                             ctypes.c_int),
    "fmmg_check": ([ctypes.c_void_p, _dp, _dp, ctypes.c_int64, _i64p, _dp, _dp, _dp], ctypes.c_int),
    "fmmg_info": ([ctypes.c_void_p, _ip, _ip, _i64p, _i64p, _ip], ctypes.c_int),
    "fmmg_stage_times": ([ctypes.c_void_p, _dp, ctypes.c_int], ctypes.c_int),
    "fmmg_setup_times": ([ctypes.c_void_p, _dp, ctypes.c_int], ctypes.c_int),
    "fmmg_set_tree_device": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "fmmg_kernel_times": ([ctypes.c_void_p, _dp, ctypes.c_int], ctypes.c_int),
    "fmmg_plan_stats": ([ctypes.c_void_p, _i64p, ctypes.c_int], ctypes.c_int),
    "fmmg_launch_count": ([ctypes.c_void_p, _i64p], ctypes.c_int),
    "fmmg_set_precision": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "fmmg_set_timing": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "fmmg_set_graph": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "fmmg_set_gemm_path": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "fmmg_autotune": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                       _dp], ctypes.c_int),
    "fmmg_tuning": ([ctypes.c_void_p, _ip, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "fmmg_device_error": ([ctypes.c_void_p, _ip], ctypes.c_int),
    "fmmg_selftest_wait": ([ctypes.c_int, ctypes.c_int, ctypes.c_int64], ctypes.c_int),
    "fmmg_graph_state": ([ctypes.c_void_p, _ip, ctypes.POINTER(ctypes.c_char_p)], ctypes.c_int),
    "fmmg_tree": ([ctypes.c_void_p, _i32p, _i64p, _i64p], ctypes.c_int),
    "fmmg_lists": ([ctypes.c_void_p, ctypes.c_int, _i64p, _i32p, _i64p], ctypes.c_int),
    "fmmg_worklist": ([ctypes.c_void_p, ctypes.c_int, _i32p, _i64p, _i32p, _i64p, _i64p], ctypes.c_int),
    "fmmg_operator": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _i64p], ctypes.c_int),
    "fmmg_dense_noalloc": ([ctypes.c_int, _dp, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "fmmg_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "fmmg_destroy": ([ctypes.c_void_p], ctypes.c_int),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FmmgError(FMMG_STATE, "libfmmg.so is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class FMM3d:
    """One evaluator: FMM3d_MPI setup()/evaluate()/check() on one GPU.

    Positions are (n, 3) float64 in the closed root box (default [0, 1]^3),
    densities (n_src, srcDOF) and values (n_trg, trgDOF), in the caller's order.
    ``device=-1`` builds the host plan only (tree, lists, operators).
    """

    def __init__(self, kernel_type=111, np_=6, pts_max=150, max_level=30, coefs=(1.0, 0.25),
                 ctr=(0.5, 0.5, 0.5), root_level=1, device=0, stream=None):
        L = lib()
        o = _Options()
        L.fmmg_default_options(ctypes.byref(o))
        o.kernel_type = kernel_type
        o.coefs[0], o.coefs[1] = coefs
        o.np, o.pts_max, o.max_level, o.root_level, o.device = np_, pts_max, max_level, root_level, device
        for d in range(3):
            o.ctr[d] = ctr[d]
        o.stream = stream
        h = ctypes.c_void_p()
        st = L.fmmg_create(ctypes.byref(o), ctypes.byref(h))
        if st != FMMG_OK:
            raise FmmgError(st, L.fmmg_last_error(None).decode())
        self.h = h
        self._stream = stream
        self.kt = kernel_type
        self.sd, self.td = KERNELS[kernel_type]
        self.ns = self.nt = 0

    def _chk(self, st):
        if st != FMMG_OK:
            raise FmmgError(st, lib().fmmg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().fmmg_destroy(self.h)
            self.h = None

    __del__ = close

    def setup(self, src, nrm=None, trg=None):
        src = _c(src).reshape(-1, 3)
        trg = src if trg is None else _c(trg).reshape(-1, 3)
        nrm = None if nrm is None else _c(nrm).reshape(-1, 3)
        self._keep = (src, trg, nrm)
        self.ns, self.nt = src.shape[0], trg.shape[0]
        self._chk(lib().fmmg_setup(self.h, self.ns, _d(src), None if nrm is None else _d(nrm), self.nt,
                                   _d(trg) if self.nt else None))

    def evaluate(self, src_den):
        """Host arrays in, host array out (copies inside), like FMM3d_MPI::evaluate."""
        den = _c(src_den).ravel()
        if den.size != self.ns * self.sd:
            raise FmmgError(FMMG_INVALID_ARG, "src_den has %d values, expected %d" % (den.size, self.ns * self.sd))
        out = np.zeros(self.nt * self.td)
        self._chk(lib().fmmg_evaluate(self.h, _d(den), _d(out)))
        return out.reshape(self.nt, self.td)

    def _order_after_torch(self):
        # a handle on its own (non-blocking) stream must not overtake torch work
        # still queued on the caller's stream (allocations, fills, copies)
        if not self._stream:
            import torch
            torch.cuda.current_stream().synchronize()

    def evaluate_device(self, den, out, k=1, precision=PREC_FP64):
        """den/out are CUDA tensors (float64, contiguous) of k right-hand sides.
        Enqueued on the handle's stream; with a handle created with stream=None
        the caller's torch stream is synchronised first."""
        self._order_after_torch()
        self._chk(lib().fmmg_evaluate_device(self.h, k, ctypes.c_void_p(den.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()), precision))

    def evaluate_stages(self, den, out, stages=STAGE_ALL, precision=PREC_FP64):
        self._order_after_torch()
        self._chk(lib().fmmg_evaluate_stages(self.h, ctypes.c_void_p(den.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()), precision, stages))

    def sync(self):
        self._chk(lib().fmmg_synchronize(self.h))

    def adjoint(self, w, src_den=None, target_grad=False, k=1):
        """Transposed evaluate on host arrays: returns (g, grad_t) with
        g = A^T w ([n_src, srcDOF], or [k, n_src, srcDOF]) and, when
        target_grad, the gradient of <w, A src_den> with respect to the target
        positions ([n_trg, 3], or [k, n_trg, 3])."""
        w = _c(w).ravel()
        if w.size != k * self.nt * self.td:
            raise FmmgError(FMMG_INVALID_ARG, "w has %d values, expected %d" % (w.size, k * self.nt * self.td))
        g = np.zeros(k * self.ns * self.sd)
        gt = np.zeros(k * 3 * self.nt) if target_grad else None
        den = None if src_den is None else _c(src_den).ravel()
        self._chk(lib().fmmg_adjoint_host(self.h, k, None if den is None else _d(den), _d(w), _d(g),
                                          None if gt is None else _d(gt)))
        shp = (self.ns, self.sd) if k == 1 else (k, self.ns, self.sd)
        gshp = (self.nt, 3) if k == 1 else (k, self.nt, 3)
        return g.reshape(shp), (None if gt is None else gt.reshape(gshp))

    def adjoint_device(self, den, w, g=None, grad_t=None, k=1):
        """fmmg_adjoint_device on CUDA tensors (float64, contiguous) of k
        right-hand sides; g and grad_t are outputs (None skips them); den is
        needed for grad_t."""
        self._order_after_torch()
        p = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        self._chk(lib().fmmg_adjoint_device(self.h, k, p(den), p(w), p(g), p(grad_t)))

    def check(self, src_den, trg_val, idx):
        """Dense FP64 GPU sums at target indices idx vs trg_val: (rel_l2, max_abs, dense)."""
        den = _c(src_den).ravel()
        val = _c(trg_val).ravel()
        idx = _c(idx, np.int64)
        rel, mx = ctypes.c_double(), ctypes.c_double()
        dense = np.zeros(idx.size * self.td)
        self._chk(lib().fmmg_check(self.h, _d(den), _d(val), idx.size, idx.ctypes.data_as(_i64p),
                                   ctypes.byref(rel), ctypes.byref(mx), _d(dense)))
        return rel.value, mx.value, dense.reshape(-1, self.td)

    def info(self):
        sd, td, md = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nn, nl = ctypes.c_int64(), ctypes.c_int64()
        self._chk(lib().fmmg_info(self.h, ctypes.byref(sd), ctypes.byref(td), ctypes.byref(nn), ctypes.byref(nl),
                                  ctypes.byref(md)))
        return dict(src_dof=sd.value, trg_dof=td.value, nodes=nn.value, leaves=nl.value, max_depth=md.value)

    def set_tree_device(self, on=True):
        """Build the octree, bin the targets and build the U/V/W/X lists on
        the GPU (the default for device handles) or on the host, from the next
        setup on."""
        self._chk(lib().fmmg_set_tree_device(self.h, 1 if on else 0))

    SETUP_PHASES = ("checks", "tree", "targets", "flags", "lists", "worklists", "adjoint_lists", "upload", "total",
                    "ops_c2e_up", "ops_c2e_down", "ops_m2m_l2l", "ops_m2l_spectra",
                    "upload_geometry", "upload_lists", "upload_operators", "upload_work")

    def setup_times(self):
        """Wall time of the last setup by phase, ms."""
        ms = np.zeros(len(self.SETUP_PHASES))
        self._chk(lib().fmmg_setup_times(self.h, _d(ms), len(ms)))
        return dict(zip(self.SETUP_PHASES, ms.tolist()))

    def stage_times(self):
        ms = np.zeros(7)
        self._chk(lib().fmmg_stage_times(self.h, _d(ms), 7))
        return dict(zip(STAGE_NAMES, ms.tolist()))

    def kernel_times(self):
        ms = np.zeros(len(KERNEL_NAMES))
        self._chk(lib().fmmg_kernel_times(self.h, _d(ms), len(KERNEL_NAMES)))
        return dict(zip(KERNEL_NAMES, ms.tolist()))

    PLAN_STATS = ("near_pairs", "s2m_pairs", "s2l_pairs", "m2t_pairs", "l2t_pairs", "v_src", "v_trg",
                  "v_parents", "v_parent_pairs", "v_interactions", "up_gemm_flops", "dn_gemm_flops", "n_eff",
                  "sdm", "tdm", "nodes", "n_eff_mixed", "up_gemm_flops_mixed", "dn_gemm_flops_mixed")
    # FLOPs counted per kernel pair for the FP64 direct sums: offset (3),
    # r^2 (5), inverse square root (1), scale and accumulate per component
    PAIR_FLOPS = {111: 11, 121: 16, 311: 40, 312: 20, 321: 36, 322: 26, 511: 40, 521: 60, 301: 46}

    def plan_stats(self):
        st = np.zeros(len(self.PLAN_STATS), dtype=np.int64)
        self._chk(lib().fmmg_plan_stats(self.h, st.ctypes.data_as(_i64p), len(self.PLAN_STATS)))
        return dict(zip(self.PLAN_STATS, st.tolist()))

    def algorithmic_work(self, k=1, precision="fp64"):
        """Per kernel class: the roofline that bounds it and its algorithmic work
        for one evaluate of k right-hand sides (pairs x FLOPs per pair x k, GEMM
        FLOPs x k, or the minimum memory bytes of the spectral M2L steps), for
        the algorithm the given form runs: the mixed form transforms on the
        (2np-1)^3 grid and folds the upward C2E into M2M for parents."""
        s = self.plan_stats()
        mm = {111: 111, 121: 111, 312: 111, 322: 111, 311: 301, 321: 301, 511: 511, 521: 511}[self.kt]
        fp, fpm = self.PAIR_FLOPS[self.kt], self.PAIR_FLOPS[mm]
        mixed = precision != "fp64"
        ne, sdm, tdm = s["n_eff_mixed" if mixed else "n_eff"], s["sdm"], s["tdm"]
        upf = s["up_gemm_flops_mixed" if mixed else "up_gemm_flops"]
        dnf = s["dn_gemm_flops_mixed" if mixed else "dn_gemm_flops"]
        cb = 16 if precision == "fp64" else 8  # bytes per complex value
        pipe = "fp64" if precision == "fp64" else "fp32"
        # a pair's kernel block is evaluated once for all k right-hand sides;
        # the multiply-add per (source, target) component repeats per one
        sd, td = KERNELS[self.kt]
        pair = fp + (k - 1) * 2 * sd * td
        pairm = fpm + (k - 1) * 2 * sdm * tdm
        return {
            "p2p_near": {"bound": pipe, "flops": s["near_pairs"] * pair, "pairs": s["near_pairs"]},
            "s2m": {"bound": pipe, "flops": s["s2m_pairs"] * pair, "pairs": s["s2m_pairs"]},
            "s2l": {"bound": pipe, "flops": s["s2l_pairs"] * pair, "pairs": s["s2l_pairs"]},
            "m2t": {"bound": pipe, "flops": s["m2t_pairs"] * pairm, "pairs": s["m2t_pairs"]},
            "l2t": {"bound": pipe, "flops": s["l2t_pairs"] * pairm, "pairs": s["l2t_pairs"]},
            "up_gemm": {"bound": pipe, "flops": k * upf},
            "dn_gemm": {"bound": pipe, "flops": k * dnf},
            "m2l_had": {"bound": pipe,
                        "bytes": cb * ne * (k * s["v_src"] * sdm + k * s["v_trg"] * tdm + 316 * sdm * tdm),
                        "flops": 8 * ne * sdm * tdm * s["v_interactions"] * k},
            "m2l_fwd": {"bound": "hbm", "bytes": k * cb * ne * s["v_src"] * sdm},
            "m2l_inv": {"bound": "hbm", "bytes": k * cb * ne * s["v_trg"] * tdm},
        }

    def launch_count(self):
        n = ctypes.c_int64()
        self._chk(lib().fmmg_launch_count(self.h, ctypes.byref(n)))
        return n.value

    def set_precision(self, precision):
        """Arithmetic of evaluate()/evaluate_host_ptr (host-buffer calls)."""
        self._chk(lib().fmmg_set_precision(self.h, precision))

    def set_timing(self, on=True):
        self._chk(lib().fmmg_set_timing(self.h, 1 if on else 0))

    def set_graph(self, on=True):
        """Replay evaluate_device as a CUDA graph (captured on the second call
        with the same k, precision and tensors)."""
        self._chk(lib().fmmg_set_graph(self.h, 1 if on else 0))

    GEMM_PATHS = {"wide": 0, "tc": 1, "narrow": 2}

    def set_gemm_path(self, path="tc"):
        """Kernels of the FP32 row GEMMs: "tc" (the tensor cores as 3xTF32,
        the default), "wide" (CUDA cores, 128 x 160 tiles) or "narrow" (CUDA
        cores, 128 x 64 tiles).  True/False mean "tc"/"wide"."""
        if path is True or path is False:
            path = "tc" if path else "wide"
        if path not in self.GEMM_PATHS:
            raise ValueError("gemm path must be one of %s" % sorted(self.GEMM_PATHS))
        self._chk(lib().fmmg_set_gemm_path(self.h, self.GEMM_PATHS[path]))

    def device_error(self):
        """1 if a kernel gave up a bounded wait since the last call (clears it)."""
        v = ctypes.c_int()
        self._chk(lib().fmmg_device_error(self.h, ctypes.byref(v)))
        return v.value

    def autotune(self, den, out, k=1, precision=PREC_FP64, reps=2):
        """Pick the launch shapes for (k, precision) by timing evaluates on
        these CUDA tensors; returns (best ms per evaluate, tuning dict)."""
        self._order_after_torch()
        ms = ctypes.c_double()
        self._chk(lib().fmmg_autotune(self.h, k, precision, ctypes.c_void_p(den.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), reps, ctypes.byref(ms)))
        return ms.value, self.tuning()

    def tuning(self, values=None):
        """Current launch shapes, or install `values` (a dict as returned)."""
        keys = ("had_rows_fp32", "had_rows_fp64", "gemm_split_ctas_per_sm", "had_fp32_rhs_per_thread",
                "tc_gemm_mask", "tc_products")
        v = (ctypes.c_int * len(keys))()
        if values is not None:
            self._chk(lib().fmmg_tuning(self.h, v, len(keys), 0))
            for i, key in enumerate(keys):
                if key in values:
                    v[i] = int(values[key])
            self._chk(lib().fmmg_tuning(self.h, v, len(keys), 1))
        self._chk(lib().fmmg_tuning(self.h, v, len(keys), 0))
        return dict(zip(keys, list(v)))

    def graph_state(self):
        act, note = ctypes.c_int(), ctypes.c_char_p()
        self._chk(lib().fmmg_graph_state(self.h, ctypes.byref(act), ctypes.byref(note)))
        return bool(act.value), (note.value or b"").decode()

    def evaluate_host_k(self, den_ptr, val_ptr, k, precision):
        """fmmg_evaluate_host: k right-hand sides on raw host pointers."""
        self._chk(lib().fmmg_evaluate_host(self.h, k, ctypes.cast(den_ptr, _dp), ctypes.cast(val_ptr, _dp),
                                           precision))

    def evaluate_host_ptr(self, den_ptr, val_ptr):
        """fmmg_evaluate on raw host pointers (e.g. pinned torch tensors)."""
        self._chk(lib().fmmg_evaluate(self.h, ctypes.cast(den_ptr, _dp), ctypes.cast(val_ptr, _dp)))

    def tree(self):
        nn = self.info()["nodes"]
        rec = np.zeros((nn, 9), dtype=np.int32)
        ps = np.zeros(max(self.ns, 1), dtype=np.int64)
        pt = np.zeros(max(self.nt, 1), dtype=np.int64)
        self._chk(lib().fmmg_tree(self.h, rec.ctypes.data_as(_i32p), ps.ctypes.data_as(_i64p),
                                  pt.ctypes.data_as(_i64p)))
        return rec, ps[: self.ns], pt[: self.nt]

    def lists(self, which):
        nn = self.info()["nodes"]
        tot = ctypes.c_int64()
        self._chk(lib().fmmg_lists(self.h, which, None, None, ctypes.byref(tot)))
        ptr = np.zeros(nn + 1, dtype=np.int64)
        idx = np.zeros(max(tot.value, 1), dtype=np.int32)
        self._chk(lib().fmmg_lists(self.h, which, ptr.ctypes.data_as(_i64p), idx.ctypes.data_as(_i32p), None))
        return ptr, idx[: tot.value]

    def worklist(self, which):
        """(rows, ptr, idx) of GPU work list `which` (fmmg_worklist); ptr and
        idx are None for the row-only lists 4 and 5, idx holds (slot,
        translation id) pairs as an [n, 2] array for 6 and 7."""
        nr, tot = ctypes.c_int64(), ctypes.c_int64()
        self._chk(lib().fmmg_worklist(self.h, which, None, None, None, ctypes.byref(nr), ctypes.byref(tot)))
        rows = np.zeros(max(nr.value, 1), dtype=np.int32)
        ptr = np.zeros(nr.value + 1, dtype=np.int64)
        idx = np.zeros(max(tot.value, 1), dtype=np.int32)
        self._chk(lib().fmmg_worklist(self.h, which, rows.ctypes.data_as(_i32p), ptr.ctypes.data_as(_i64p),
                                      idx.ctypes.data_as(_i32p), None, None))
        if which in (4, 5):
            return rows[: nr.value], None, None
        if which >= 6:
            return rows[: nr.value], ptr, idx[: tot.value].reshape(-1, 2)
        return rows[: nr.value], ptr, idx[: tot.value]

    def operator(self, which, idx=0):
        n = ctypes.c_int64()
        self._chk(lib().fmmg_operator(self.h, which, idx, None, None, ctypes.byref(n)))
        out = np.zeros(n.value)
        self._chk(lib().fmmg_operator(self.h, which, idx, _d(out), None, None))
        return out

    def set_operator(self, which, idx, values):
        v = _c(values).ravel()
        self._chk(lib().fmmg_operator(self.h, which, idx, None, _d(v), None))
