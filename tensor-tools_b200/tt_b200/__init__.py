"""Python binding of the B200 two-site DMRG C ABI (include/tt_b200.h, include/tt_dmrg.h).

The binding is a thin ctypes layer: every object lives in the C++ host layer
of ``lib/libtt_b200.so`` and every number is computed by its sm_100a kernels.
There is no CPU fallback -- importing works without a GPU (the library only
needs the CUDA runtime to load), but creating a ``Context`` requires a B200.

Names follow tensor-tools: ``QTensor`` (qtensor), ``BigQTensor``
(big_qtensor), ``svd``/``svd_bond``, ``QMPS``/``QMPO``, ``QDMRG`` (the
schedule overload of ``dmrg``).
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "lib", "libtt_b200.so")
HEADERS = [os.path.join(ROOT, "include", "tt_b200.h"), os.path.join(ROOT, "include", "tt_dmrg.h")]

TT_OK = 0
TT_ERR_TIMEOUT = 4  # a bounded device wait gave up (include/tt_b200.h)
MoveFromLeft, MoveFromRight = 0, 1
Inward, Outward = 0, 1
Link, Site = 0, 1


class TTError(RuntimeError):
    pass


TT_PREC_FP64, TT_PREC_TF32, TT_PREC_TF32X3, TT_PREC_TF32_AUTO, TT_PREC_TF32X3_AUTO = 0, 1, 2, 3, 4
# "*-auto": per contraction, the tensor-core kind where the plan's cost model
# predicts it faster than FP64, FP64 elsewhere
PRECISIONS = {"fp64": TT_PREC_FP64, "tf32": TT_PREC_TF32, "tf32x3": TT_PREC_TF32X3,
              "tf32-auto": TT_PREC_TF32_AUTO, "tf32x3-auto": TT_PREC_TF32X3_AUTO}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libtt_b200.so not built: run tensor-tools_b200/build.py (%s)" % LIB_PATH)
    return C.CDLL(LIB_PATH)


lib = _load()

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
D = C.c_double
PI32 = C.POINTER(C.c_int32)
PI64 = C.POINTER(C.c_int64)
PD = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)


class IndexDesc(C.Structure):
    _fields_ = [("arrow", I32), ("type", I32), ("level", I32), ("n_sectors", I32),
                ("name", C.c_char_p), ("qn", PI32), ("qdim", PI32)]


def _proto(name, *args):
    f = getattr(lib, name)
    f.restype = C.c_int
    f.argtypes = list(args)
    return f


_proto("tt_ctx_create", C.c_int, PP)
_proto("tt_ctx_destroy", P)
_proto("tt_ctx_synchronize", P)
_proto("tt_ctx_stream", P, PP)
_proto("tt_ctx_wait_stats", P, PD, PI64)
_proto("tt_ctx_pool_trims", P, PI64)
_proto("tt_ctx_alloc_stats", P, PD, PD, PD, PD, PI64, PI64, PI64, C.c_int)
_proto("tt_ctx_set_block_cache", P, C.c_int64)
_proto("tt_ctx_launch_count", P, PI64)
lib.tt_get_last_error.restype = C.c_char_p
lib.tt_get_last_error.argtypes = []
_proto("tt_dmrg_bind", P)
_proto("tt_dmrg_set_precision", C.c_int, C.c_int, C.c_int)
_proto("tt_dmrg_set_davidson", C.c_int)
_proto("tt_dmrg_set_profile_step", C.c_int)
_proto("tt_dmrg_davidson_fallbacks", PI64)
_proto("tt_dmrg_davidson_refills", PI64)
_proto("tt_plan_device_status", P, P, C.POINTER(C.c_int))
_proto("tt_dmrg_unbind")
_proto("tt_device_alloc", P, C.c_size_t, PP)
_proto("tt_device_free", P, P)
_proto("tt_memcpy_h2d", P, P, P, C.c_size_t)
_proto("tt_memcpy_d2h", P, P, P, C.c_size_t)
_proto("tt_memset_zero", P, P, C.c_size_t)
_proto("tt_vec_dot", P, I64, P, P, P)
_proto("tt_vec_nrm2", P, I64, P, P)
_proto("tt_vec_axpy", P, I64, D, P, P)
_proto("tt_vec_scal", P, I64, D, P)
_proto("tt_vec_multidot", P, I64, C.c_int, PP, P, P)
_proto("tt_vec_lincomb_dev", P, I64, C.c_int, PP, P, D, C.c_int, P)
_proto("tt_vec_fill_random", P, I64, P, C.c_int, P, C.c_uint64)
_proto("tt_vec_precondition", P, I64, P, P, D)
_proto("tt_qtensor_create", C.c_int, C.POINTER(IndexDesc), PP)
_proto("tt_qtensor_init_blocks", P)
_proto("tt_qtensor_set_blocks", P, C.c_int, PI32)
_proto("tt_qtensor_destroy", P)
_proto("tt_qtensor_copy", P, PP)
_proto("tt_qtensor_rank", P, C.POINTER(C.c_int))
_proto("tt_qtensor_index", P, C.c_int, PI32, PI32, PI32, PI32, C.c_char_p, C.c_int, PI32, PI32, C.c_int)
_proto("tt_qtensor_num_blocks", P, C.POINTER(C.c_int))
_proto("tt_qtensor_block_info", P, C.c_int, PI32, PI32, PI32, PI64)
_proto("tt_qtensor_find_block", P, PI32, C.POINTER(C.c_int))
_proto("tt_qtensor_get_block", P, C.c_int, PD)
_proto("tt_qtensor_set_block", P, C.c_int, PD)
_proto("tt_qtensor_prime", P, C.c_int)
_proto("tt_qtensor_dag", P)
_proto("tt_qtensor_contract", P, P, PP)
_proto("tt_qtensor_norm", P, PD)
_proto("tt_qtensor_scale", P, D)
_proto("tt_qtensor_add", P, P, D)
_proto("tt_qtensor_inner_product", P, P, PD)
_proto("tt_qtensor_svd", P, C.c_int, C.POINTER(C.c_int), C.c_int, D, C.c_uint, PP, PP, PP, PD,
       C.POINTER(C.c_uint))
_proto("tt_qtensor_svd_bond", P, P, P, C.c_int, C.c_int, D, C.c_ulong, PP, PD, C.POINTER(C.c_uint))
_proto("tt_qtensor_svd_bond_sectors", P, P, P, C.c_int, C.c_int, D, C.c_ulong, PP, PD, C.POINTER(C.c_uint),
       C.POINTER(C.c_int), PI32, C.POINTER(C.c_uint32), C.c_int)
_proto("tt_qtensor_env_update", P, P, P, PP)
_proto("tt_bigq_create", P, P, P, P, PP)
_proto("tt_bigq_product", P, P, PP)
_proto("tt_bigq_size", P, C.POINTER(C.c_uint64))
_proto("tt_bigq_davidson", P, P, C.c_int, D, PD, C.POINTER(C.c_int))
_proto("tt_bigq_destroy", P)
_proto("tt_qmps_product_spinhalf", C.c_int, C.POINTER(C.c_int), C.c_uint, PP)
_proto("tt_qmps_destroy", P)
_proto("tt_qmps_length", P, C.POINTER(C.c_int))
_proto("tt_qmps_bond_dims", P, C.POINTER(C.c_int))
_proto("tt_qmps_center", P, C.POINTER(C.c_int))
_proto("tt_qmps_position", P, C.c_int)
_proto("tt_qmps_tensor", P, C.c_int, PP)
_proto("tt_qmps_data_size", P, PI64)
_proto("tt_qmps_get_data", P, PD)
_proto("tt_qmps_set_data", P, PD)
_proto("tt_qmps_sites_size", P, C.c_int, C.c_int, C.POINTER(I64))
_proto("tt_qmps_get_sites", P, C.c_int, C.c_int, PD)
_proto("tt_qmps_set_sites", P, C.c_int, C.c_int, PD)
_proto("tt_qdmrg_env", P, C.c_int, C.c_int, PP)
_proto("tt_dmps_product_spinhalf", C.c_int, C.POINTER(C.c_int), C.c_uint, PP)
_proto("tt_dmps_destroy", P)
_proto("tt_dmps_bond_dims", P, C.POINTER(C.c_int))
_proto("tt_dmpo_heisenberg", C.c_int, PD, D, C.c_uint, PP)
_proto("tt_dmpo_destroy", P)
_proto("tt_ddmrg_run", P, P, C.c_int, C.POINTER(C.c_int), C.c_int, PD, C.c_int, C.POINTER(C.c_int), C.c_int,
       PD, PD, C.POINTER(C.c_int))
_proto("tt_qmpo_heisenberg", C.c_int, PD, D, C.c_uint, PP)
_proto("tt_autompo_create", PP)
_proto("tt_autompo_destroy", P)
_proto("tt_autompo_add", P, D, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int))
_proto("tt_autompo_size", P, C.POINTER(C.c_int))
_proto("tt_autompo_term", P, C.c_int, PD, C.POINTER(C.c_int), C.c_char_p, C.POINTER(C.c_int), C.c_int)
_proto("tt_autompo_link_dims", P, C.c_int, C.c_int, C.POINTER(C.c_int))
_proto("tt_qmpo_from_autompo", P, C.c_int, C.c_uint, PP)
_proto("tt_dmpo_from_autompo", P, C.c_int, C.c_uint, PP)
_proto("tt_dmpo_tensor", P, C.c_int, PI64, PD, I64)
for _pre in ("tt_qmps", "tt_dmps"):
    _proto(_pre + "_save", P, C.c_char_p, C.c_char_p)
    _proto(_pre + "_length", P, C.POINTER(C.c_int))
    _proto(_pre + "_load", C.c_char_p, C.c_char_p, PP)
    _proto(_pre + "_overlap", P, P, PD)
    _proto(_pre + "_expectation", P, P, P, PD)
    _proto(_pre + "_measure_sz", P, PD, PD)
_proto("tt_qmpo_destroy", P)
_proto("tt_qmpo_tensor", P, C.c_int, PP)
_proto("tt_qdmrg_create", P, P, PP)
_proto("tt_ctx_device_status", P, C.POINTER(C.c_int))
_proto("tt_ctx_clear_device_status", P)
_proto("tt_ctx_set_wait_limit", P, I64)
_proto("tt_ctx_memory", P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.c_int)
_proto("tt_vec_scale_mode", P, I64, C.c_int, I64, PD, P)
_proto("tt_qdmrg_sweep", P, C.c_int, D, C.c_int, PD)
_proto("tt_qdmrg_set_noise", P, D)
_proto("tt_qdmrg_finish", P)
_proto("tt_qdmrg_walk", P, C.c_int, C.c_int, D, C.c_int, PD)
_proto("tt_qdmrg_position", P, C.POINTER(C.c_int))
_proto("tt_qdmrg_destroy", P)
_proto("tt_qdmrg_run", P, P, C.c_int, C.POINTER(C.c_int), C.c_int, PD, C.c_int, C.POINTER(C.c_int),
       C.c_int, PD, PP)
_proto("tt_qdmrg_num_steps", P, C.POINTER(C.c_int))
_proto("tt_qdmrg_step", P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), PD, PD, C.POINTER(C.c_uint),
       C.POINTER(C.c_int), PD)
_proto("tt_qdmrg_step_sectors", P, C.c_int, C.POINTER(C.c_int), PI32, C.POINTER(C.c_uint32), C.c_int)
_proto("tt_qdmrg_stats", P, PD, PD, PD)
_proto("tt_qdmrg_step_profile", P, C.c_int, C.POINTER(C.c_int), PD, PD, PD, PD)
_proto("tt_qdmrg_step_device_ms", P, C.c_int, PD, PD, PD, PD)
_proto("tt_dmrg_set_profiling", C.c_int)
_proto("tt_dmrg_planning_counters", PD, PI64, PD, PI64)
_proto("tt_dmrg_cache_stats", PI64, PI64, PI64, PI64)
_proto("tt_contract_plan_timers", PD, C.c_int)
_proto("tt_eig_redo_count", P, PI64)
_proto("tt_dmrg_heff_parts", PD, PD, PD)
_proto("tt_sym_eig_batched", P, C.c_void_p, C.c_int, P, P, P, P)
_proto("tt_qdmrg_num_sweeps", P, C.POINTER(C.c_int))
_proto("tt_qdmrg_sweep_info", P, C.c_int, PD, PD)


def _chk(rc, what=""):
    if rc != TT_OK:
        msg = lib.tt_get_last_error().decode(errors="replace")
        raise TTError("%s failed (status %d): %s" % (what, rc, msg))


def declared_symbols() -> List[str]:
    """Every entry point the public headers declare."""
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(?:int|const char\*)\s+(tt_\w+)\s*\(", src)
    return sorted(set(names))


class Context:
    """One device context (stream, pool); binds itself to the calling thread."""

    def __init__(self, device: int = 0):
        self.h = P()
        _chk(lib.tt_ctx_create(device, C.byref(self.h)), "tt_ctx_create")
        _chk(lib.tt_dmrg_bind(self.h), "tt_dmrg_bind")

    def sync(self):
        _chk(lib.tt_ctx_synchronize(self.h), "sync")

    def stream(self) -> int:
        s = P()
        _chk(lib.tt_ctx_stream(self.h, C.byref(s)), "stream")
        return s.value or 0

    def wait_stats(self):
        """(host seconds blocked in stream synchronisations, number of them)."""
        s, n = D(), I64()
        _chk(lib.tt_ctx_wait_stats(self.h, C.byref(s), C.byref(n)), "wait stats")
        return s.value, n.value

    def pool_trims(self) -> int:
        """Pool allocations that failed once and were retried after a trim."""
        n = I64()
        _chk(lib.tt_ctx_pool_trims(self.h, C.byref(n)), "pool trims")
        return n.value

    def alloc_stats(self, reset_max: bool = False) -> dict:
        """Host seconds inside device-pool allocate / free calls: totals, the
        largest single call since the last reset, and the allocation count."""
        a, am, f, fm, n, hits, cached = D(), D(), D(), D(), I64(), I64(), I64()
        _chk(lib.tt_ctx_alloc_stats(self.h, C.byref(a), C.byref(am), C.byref(f), C.byref(fm), C.byref(n),
                                    C.byref(hits), C.byref(cached), int(reset_max)), "alloc stats")
        return {"alloc_s": a.value, "alloc_max_s": am.value, "free_s": f.value, "free_max_s": fm.value,
                "allocs": n.value, "cache_hits": hits.value, "cached_bytes": cached.value}

    def set_block_cache(self, nbytes: int):
        """Bytes of freed large blocks the context keeps for reuse (0: off)."""
        _chk(lib.tt_ctx_set_block_cache(self.h, int(nbytes)), "block cache")

    def launches(self) -> int:
        n = I64()
        _chk(lib.tt_ctx_launch_count(self.h, C.byref(n)), "launch count")
        return n.value

    def device_status(self) -> int:
        """TT_OK, or TT_ERR_TIMEOUT once a bounded tensor-core wait gave up (synchronises)."""
        n = C.c_int()
        _chk(lib.tt_ctx_device_status(self.h, C.byref(n)), "device status")
        return n.value

    def clear_device_status(self):
        _chk(lib.tt_ctx_clear_device_status(self.h), "clear device status")

    def memory(self, reset_high: bool = False):
        """Pool bytes: (in use, high-water mark of use, reserved from the device)."""
        u, h, r = I64(), I64(), I64()
        _chk(lib.tt_ctx_memory(self.h, C.byref(u), C.byref(h), C.byref(r), int(reset_high)), "memory")
        return u.value, h.value, r.value

    def set_wait_limit(self, polls: int):
        """Test hook: polls of the tensor-core kernels' main-loop waits (< 0: the default)."""
        _chk(lib.tt_ctx_set_wait_limit(self.h, polls), "set wait limit")

    def close(self):
        if self.h:
            lib.tt_dmrg_unbind()
            lib.tt_ctx_destroy(self.h)
            self.h = P()


# ---------------------------------------------------------------------------
# qtensor handles <-> oracle-style numpy block tensors
# ---------------------------------------------------------------------------
class QTensor:
    """Handle of a device qtensor (qtensor/qtensor.h:47-164)."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib.tt_qtensor_destroy(self.h)
            except Exception:
                pass
            self.h = None

    @staticmethod
    def _descs(indices):
        keep = []
        descs = (IndexDesc * len(indices))()
        for i, ix in enumerate(indices):
            qn = np.array([v for (q, _) in ix.qns for v in q], dtype=np.int32)
            qd = np.array([d for (_, d) in ix.qns], dtype=np.int32)
            name = ix.name.encode()
            keep += [qn, qd, name]
            descs[i] = IndexDesc(ix.arrow, ix.type, ix.level, len(ix.qns), name,
                                 qn.ctypes.data_as(PI32), qd.ctypes.data_as(PI32))
        return descs, keep

    @classmethod
    def create(cls, indices, init_blocks: bool = True) -> "QTensor":
        descs, keep = cls._descs(indices)
        h = P()
        _chk(lib.tt_qtensor_create(len(indices), descs, C.byref(h)), "tt_qtensor_create")
        t = cls(h)
        if init_blocks:
            _chk(lib.tt_qtensor_init_blocks(h), "init_blocks")
        return t

    @classmethod
    def from_oracle(cls, T) -> "QTensor":
        descs, keep = cls._descs(T.idx)
        h = P()
        _chk(lib.tt_qtensor_create(T.rank, descs, C.byref(h)), "tt_qtensor_create")
        t = cls(h)
        qi = np.array([p for q in T.bqi for p in q], dtype=np.int32)
        _chk(lib.tt_qtensor_set_blocks(h, len(T.blocks), qi.ctypes.data_as(PI32)), "set_blocks")
        for b, blk in enumerate(T.blocks):
            data = np.asfortranarray(blk).ravel(order="F").astype(np.float64)
            _chk(lib.tt_qtensor_set_block(h, b, data.ctypes.data_as(PD)), "set_block")
        return t

    @property
    def rank(self) -> int:
        r = C.c_int()
        _chk(lib.tt_qtensor_rank(self.h, C.byref(r)), "rank")
        return r.value

    def index_info(self, i):
        a, t, l, n = I32(), I32(), I32(), I32()
        name = C.create_string_buffer(256)
        cap = 512
        qn = (I32 * (2 * cap))()
        qd = (I32 * cap)()
        _chk(lib.tt_qtensor_index(self.h, i, C.byref(a), C.byref(t), C.byref(l), C.byref(n), name, 256,
                                  qn, qd, cap), "index")
        sectors = [((qn[2 * s], qn[2 * s + 1]), qd[s]) for s in range(n.value)]
        return dict(arrow=a.value, type=t.value, level=l.value, name=name.value.decode(), qns=sectors)

    def num_blocks(self) -> int:
        n = C.c_int()
        _chk(lib.tt_qtensor_num_blocks(self.h, C.byref(n)), "num_blocks")
        return n.value

    def blocks(self):
        """[(qn tuple, qi tuple, ndarray)] with axes in the tensor's index order."""
        r = self.rank
        out = []
        for b in range(self.num_blocks()):
            qn = (I32 * (2 * r))()
            qi = (I32 * r)()
            qd = (I32 * r)()
            sz = I64()
            _chk(lib.tt_qtensor_block_info(self.h, b, qn, qi, qd, C.byref(sz)), "block_info")
            data = np.empty(sz.value, dtype=np.float64)
            _chk(lib.tt_qtensor_get_block(self.h, b, data.ctypes.data_as(PD)), "get_block")
            dims = tuple(qd[j] for j in range(r))
            out.append((tuple((qn[2 * j], qn[2 * j + 1]) for j in range(r)),
                        tuple(qi[j] for j in range(r)), data.reshape(dims, order="F")))
        return out

    def to_oracle(self):
        from oracle.qtensor import QIndex, QTensor as OQ
        idx = []
        for i in range(self.rank):
            inf = self.index_info(i)
            ix = QIndex(inf["arrow"], inf["name"], inf["type"], inf["level"])
            ix.qns = list(inf["qns"])
            idx.append(ix)
        T = OQ(idx)
        T.initted = True
        for qn, qi, data in self.blocks():
            T._append_block(qn, qi, data.shape, data.copy())
        return T

    def copy(self) -> "QTensor":
        h = P()
        _chk(lib.tt_qtensor_copy(self.h, C.byref(h)), "copy")
        return QTensor(h)

    def prime(self, inc=1):
        _chk(lib.tt_qtensor_prime(self.h, inc), "prime")

    def dag(self):
        _chk(lib.tt_qtensor_dag(self.h), "dag")

    def __mul__(self, other: "QTensor") -> "QTensor":
        h = P()
        _chk(lib.tt_qtensor_contract(self.h, other.h, C.byref(h)), "contract")
        return QTensor(h)

    def norm(self) -> float:
        v = D()
        _chk(lib.tt_qtensor_norm(self.h, C.byref(v)), "norm")
        return v.value

    def scale(self, c: float):
        _chk(lib.tt_qtensor_scale(self.h, c), "scale")

    def add(self, other: "QTensor", c: float = 1.0):
        _chk(lib.tt_qtensor_add(self.h, other.h, c), "add")

    def inner_product(self, other: "QTensor") -> float:
        v = D()
        _chk(lib.tt_qtensor_inner_product(self.h, other.h, C.byref(v)), "inner_product")
        return v.value


def svd(A: QTensor, left_axes: Sequence[int], direction: int, cutoff: float = 0.0, K: int = 0):
    """svd(A, left, right, U, V, S, direction, cutoff, K) -> (U, V, S, trunc_err, kept)."""
    la = (C.c_int * len(left_axes))(*left_axes)
    U, V, S = P(), P(), P()
    te = D()
    kept = C.c_uint()
    _chk(lib.tt_qtensor_svd(A.h, len(left_axes), la, direction, cutoff, K, C.byref(U), C.byref(V),
                            C.byref(S), C.byref(te), C.byref(kept)), "svd")
    return QTensor(U), QTensor(V), QTensor(S), te.value, kept.value


def svd_bond(combined: QTensor, A_left: QTensor, A_right: QTensor, mid_axis: int, direction: int,
             cutoff: float = 0.0, K: int = 0):
    S = P()
    te = D()
    kept = C.c_uint()
    _chk(lib.tt_qtensor_svd_bond(combined.h, A_left.h, A_right.h, mid_axis, direction, cutoff, K, C.byref(S),
                                 C.byref(te), C.byref(kept)), "svd_bond")
    return QTensor(S), te.value, kept.value


def svd_bond_sectors(combined: QTensor, A_left: QTensor, A_right: QTensor, mid_axis: int, direction: int,
                     cutoff: float = 0.0, K: int = 0):
    """svd_bond plus its mid-QN sectors: (S, trunc_err, kept, [(qn, kept_in_sector), ...])."""
    S = P()
    te = D()
    kept = C.c_uint()
    n = C.c_int()
    cap = 256
    qn = (C.c_int32 * (2 * cap))()
    ks = (C.c_uint32 * cap)()
    _chk(lib.tt_qtensor_svd_bond_sectors(combined.h, A_left.h, A_right.h, mid_axis, direction, cutoff, K,
                                         C.byref(S), C.byref(te), C.byref(kept), C.byref(n), qn, ks, cap),
         "svd_bond_sectors")
    if n.value > cap:
        raise TTError("svd_bond_sectors: more than %d sectors" % cap)
    return QTensor(S), te.value, kept.value, [((qn[2 * j], qn[2 * j + 1]), ks[j]) for j in range(n.value)]


def env_update(env: QTensor, A: QTensor, W: QTensor) -> QTensor:
    """One environment step ((A^dag' env) W) A (algos/dmrg/dmrg.cpp:491-509)."""
    h = P()
    _chk(lib.tt_qtensor_env_update(env.h, A.h, W.h, C.byref(h)), "env_update")
    return QTensor(h)


class BigQTensor:
    """big_qtensor: L, pre-contracted W1*W2 and R (qtensor/big_qtensor.{h,cpp})."""

    def __init__(self, L: QTensor, W1: QTensor, W2: Optional[QTensor], R: QTensor):
        self.h = P()
        _chk(lib.tt_bigq_create(L.h, W1.h, W2.h if W2 is not None else None, R.h, C.byref(self.h)), "bigq")

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_bigq_destroy(self.h)
            self.h = None

    def product(self, v: QTensor) -> QTensor:
        h = P()
        _chk(lib.tt_bigq_product(self.h, v.h, C.byref(h)), "product")
        return QTensor(h)

    def size(self) -> int:
        s = C.c_uint64()
        _chk(lib.tt_bigq_size(self.h, C.byref(s)), "size")
        return s.value

    def davidson(self, x: QTensor, max_restart: int, tol: float = 1e-12) -> Tuple[float, int]:
        e = D()
        mv = C.c_int()
        _chk(lib.tt_bigq_davidson(self.h, x.h, max_restart, tol, C.byref(e), C.byref(mv)), "davidson")
        return e.value, mv.value


class QMPS:
    def __init__(self, L: int, state: Sequence[int] = None, mps_id: int = 1, _handle=None):
        self.L = L
        self.h = P()
        if _handle is not None:
            self.h = _handle
            return
        st = (C.c_int * L)(*state)
        _chk(lib.tt_qmps_product_spinhalf(L, st, mps_id, C.byref(self.h)), "qmps")

    def save(self, fn: str, wfn: Optional[str] = None):
        """qTensorTrain::save: metadata to fn + '.ttmps', blocks to wfn (default fn + '__T.bin')."""
        _chk(lib.tt_qmps_save(self.h, fn.encode(), wfn.encode() if wfn else None), "qmps save")

    @classmethod
    def load(cls, fn: str, data_prefix: str = "") -> "QMPS":
        """qTensorTrain::load(fn, dataPrefix) from a '.ttmps' metadata file."""
        h = P()
        _chk(lib.tt_qmps_load(fn.encode(), data_prefix.encode(), C.byref(h)), "qmps load")
        n = C.c_int()
        _chk(lib.tt_qmps_length(h, C.byref(n)), "qmps length")
        return cls(n.value, _handle=h)

    def overlap(self, other=None) -> float:
        """psiphi(self, other) (mps/observables.cpp:382-450); other defaults to self."""
        out = D()
        _chk(lib.tt_qmps_overlap(self.h, (other or self).h, C.byref(out)), "overlap")
        return out.value

    def expectation(self, H, other=None) -> float:
        """psiHphi(self, H, other) (mps/observables.cpp:25-103), unnormalised."""
        out = D()
        _chk(lib.tt_qmps_expectation(self.h, H.h, (other or self).h, C.byref(out)), "expectation")
        return out.value

    def measure_sz(self):
        """(<Sz_i> as an (L,) array, <Sz_i Sz_j> as an (L, L) array), normalised by <psi|psi>."""
        sz = np.zeros(self.L)
        szsz = np.zeros((self.L, self.L))
        _chk(lib.tt_qmps_measure_sz(self.h, sz.ctypes.data_as(PD), szsz.ctypes.data_as(PD)), "measure_sz")
        return sz, szsz

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_qmps_destroy(self.h)
            self.h = None

    def bond_dims(self) -> List[int]:
        out = (C.c_int * (self.L + 1))()
        _chk(lib.tt_qmps_bond_dims(self.h, out), "bond_dims")
        return list(out)

    def center(self) -> int:
        c = C.c_int()
        _chk(lib.tt_qmps_center(self.h, C.byref(c)), "center")
        return c.value

    def position(self, site: int):
        _chk(lib.tt_qmps_position(self.h, site), "position")

    def tensor(self, i: int) -> QTensor:
        h = P()
        _chk(lib.tt_qmps_tensor(self.h, i, C.byref(h)), "qmps tensor")
        return QTensor(h)

    def data_size(self) -> int:
        n = I64()
        _chk(lib.tt_qmps_data_size(self.h, C.byref(n)), "data_size")
        return n.value

    def get_data(self, host: np.ndarray):
        """All block data into ``host`` (float64, data_size() elements; pin it for bandwidth)."""
        _chk(lib.tt_qmps_get_data(self.h, host.ctypes.data_as(PD)), "get_data")

    def set_data(self, host: np.ndarray):
        _chk(lib.tt_qmps_set_data(self.h, host.ctypes.data_as(PD)), "set_data")

    def sites_size(self, first: int, last: int) -> int:
        """Elements of the site tensors [first, last)."""
        n = I64()
        _chk(lib.tt_qmps_sites_size(self.h, first, last, C.byref(n)), "sites_size")
        return n.value

    def get_sites(self, first: int, last: int, host: np.ndarray):
        """Blocks of the site tensors [first, last) into host (float64, pinned for full bandwidth)."""
        _chk(lib.tt_qmps_get_sites(self.h, first, last, host.ctypes.data_as(PD)), "get_sites")

    def set_sites(self, first: int, last: int, host: np.ndarray):
        _chk(lib.tt_qmps_set_sites(self.h, first, last, host.ctypes.data_as(PD)), "set_sites")


class QMPO:
    """U(1) qMPO: the hand-written Heisenberg chain (models/hams/Heisenberg.cpp:333-402),
    or any spin-1/2 AutoMPO through ``QMPO.from_autompo``."""

    def __init__(self, L: int, dh: Optional[Sequence[float]] = None, tE: float = 0.0, mpo_id: int = 2,
                 _handle=None):
        self.L = L
        self.h = P()
        if _handle is not None:
            self.h = _handle
            return
        arr = (D * L)(*dh) if dh is not None else None
        _chk(lib.tt_qmpo_heisenberg(L, arr, tE, mpo_id, C.byref(self.h)), "qmpo")

    @classmethod
    def from_autompo(cls, ampo: "AutoMPO", N: int, mpo_id: int = 2) -> "QMPO":
        h = P()
        _chk(lib.tt_qmpo_from_autompo(ampo.h, N, mpo_id, C.byref(h)), "qmpo from autompo")
        return cls(N, _handle=h)

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_qmpo_destroy(self.h)
            self.h = None

    def tensor(self, i: int) -> QTensor:
        h = P()
        _chk(lib.tt_qmpo_tensor(self.h, i, C.byref(h)), "qmpo tensor")
        return QTensor(h)


class QDMRG:
    """Step-wise driver of dmrg(psi, H, nsweeps, maxm[], cutoff[], max_restart[])."""

    def __init__(self, psi: QMPS, H: QMPO):
        self.psi, self.H = psi, H
        self.h = P()
        _chk(lib.tt_qdmrg_create(psi.h, H.h, C.byref(self.h)), "qdmrg create")

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_qdmrg_destroy(self.h)
            self.h = None

    def sweep(self, max_bd: int, cutoff: float, max_restart: int, noise: float = 0.0) -> float:
        """One sweep; noise > 0 adds the density-matrix perturbation to its truncations."""
        _chk(lib.tt_qdmrg_set_noise(self.h, noise), "set_noise")
        e = D()
        _chk(lib.tt_qdmrg_sweep(self.h, max_bd, cutoff, max_restart, C.byref(e)), "sweep")
        return e.value

    def finish(self):
        _chk(lib.tt_qdmrg_finish(self.h), "finish")

    def walk(self, to_site: int, max_bd: int, cutoff: float, max_restart: int, noise: float = 0.0) -> float:
        """Two-site updates moving the orthogonality centre to to_site (0-based);
        returns the last step's energy.  Sweeps need the centre back at 0."""
        _chk(lib.tt_qdmrg_set_noise(self.h, noise), "set_noise")
        e = D()
        _chk(lib.tt_qdmrg_walk(self.h, to_site, max_bd, cutoff, max_restart, C.byref(e)), "walk")
        return e.value

    def position(self) -> int:
        n = C.c_int()
        _chk(lib.tt_qdmrg_position(self.h, C.byref(n)), "position")
        return n.value

    def run(self, nsweeps, maxm, cutoff, max_restart, start_sweep: int = 0, noise=None) -> float:
        """Sweeps start_sweep .. nsweeps-1 of the schedule (maxm[s % len] ...),
        then the final position(0); start_sweep > 0 resumes a loaded checkpoint.
        noise: per-sweep noise values (the last one repeats), default none."""
        e = 0.0
        for s in range(start_sweep, nsweeps):
            nz = 0.0 if not noise else noise[min(s, len(noise) - 1)]
            e = self.sweep(maxm[s % len(maxm)], cutoff[s % len(cutoff)], max_restart[s % len(max_restart)], nz)
        self.finish()
        return e

    def steps(self):
        n = C.c_int()
        _chk(lib.tt_qdmrg_num_steps(self.h, C.byref(n)), "num_steps")
        out = []
        for i in range(n.value):
            site, d, mv = C.c_int(), C.c_int(), C.c_int()
            e, te, fl = D(), D(), D()
            kept = C.c_uint()
            _chk(lib.tt_qdmrg_step(self.h, i, C.byref(site), C.byref(d), C.byref(e), C.byref(te),
                                   C.byref(kept), C.byref(mv), C.byref(fl)), "step")
            ns = C.c_int()
            cap = 256
            qn = (I32 * (2 * cap))()
            kp = (C.c_uint32 * cap)()
            _chk(lib.tt_qdmrg_step_sectors(self.h, i, C.byref(ns), qn, kp, cap), "step sectors")
            sec = tuple(((qn[2 * j], qn[2 * j + 1]), kp[j]) for j in range(min(ns.value, cap)))
            out.append(dict(site=site.value, direction=d.value, energy=e.value, trunc_err=te.value,
                            kept=kept.value, matvecs=mv.value, heff_flops=fl.value, sectors=sec))
        return out

    def profile(self):
        """Per step: (largest SVD sector, Davidson s, SVD s, env-update s)."""
        n = C.c_int()
        _chk(lib.tt_qdmrg_num_steps(self.h, C.byref(n)), "num_steps")
        out = []
        for i in range(n.value):
            g = C.c_int()
            a, b, c, e = D(), D(), D(), D()
            _chk(lib.tt_qdmrg_step_profile(self.h, i, C.byref(g), C.byref(a), C.byref(b), C.byref(c), C.byref(e)),
                 "profile")
            out.append((g.value, a.value, b.value, c.value, e.value))
        return out

    def device_profile(self, first: int = 0):
        """Per step from `first` on: device-stream milliseconds of (Davidson,
        SVD, env update, gap since the previous step's end), event-timed."""
        n = C.c_int()
        _chk(lib.tt_qdmrg_num_steps(self.h, C.byref(n)), "num_steps")
        out = []
        for i in range(first, n.value):
            a, b, c, g = D(), D(), D(), D()
            _chk(lib.tt_qdmrg_step_device_ms(self.h, i, C.byref(a), C.byref(b), C.byref(c), C.byref(g)),
                 "device profile")
            out.append((a.value, b.value, c.value, g.value))
        return out

    def env(self, which: int, i: int) -> QTensor:
        """Copy of TL[i] (which=0) or TR[i] (which=1)."""
        h = P()
        _chk(lib.tt_qdmrg_env(self.h, which, i, C.byref(h)), "env")
        return QTensor(h)

    def stats(self):
        f, s, e0 = D(), D(), D()
        _chk(lib.tt_qdmrg_stats(self.h, C.byref(f), C.byref(s), C.byref(e0)), "stats")
        return dict(heff_flops=f.value, heff_seconds=s.value, initial_energy=e0.value)

    def sweeps(self):
        n = C.c_int()
        _chk(lib.tt_qdmrg_num_sweeps(self.h, C.byref(n)), "num_sweeps")
        out = []
        for i in range(n.value):
            e, s = D(), D()
            _chk(lib.tt_qdmrg_sweep_info(self.h, i, C.byref(e), C.byref(s)), "sweep info")
            out.append((e.value, s.value))
        return out


# ---------------------------------------------------------------------------
# dense (dtensor) path
# ---------------------------------------------------------------------------
class DMPS:
    """MPS(sites, product string) of the dense path (mps/tt.cpp:225-262)."""

    def __init__(self, L: int, state: Sequence[int] = None, mps_id: int = 1, _handle=None):
        self.L = L
        self.h = P()
        if _handle is not None:
            self.h = _handle
            return
        _chk(lib.tt_dmps_product_spinhalf(L, (C.c_int * L)(*state), mps_id, C.byref(self.h)), "dmps")

    def save(self, fn: str, wfn: Optional[str] = None):
        _chk(lib.tt_dmps_save(self.h, fn.encode(), wfn.encode() if wfn else None), "dmps save")

    @classmethod
    def load(cls, fn: str, data_prefix: str = "") -> "DMPS":
        h = P()
        _chk(lib.tt_dmps_load(fn.encode(), data_prefix.encode(), C.byref(h)), "dmps load")
        n = C.c_int()
        _chk(lib.tt_dmps_length(h, C.byref(n)), "dmps length")
        return cls(n.value, _handle=h)

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_dmps_destroy(self.h)
            self.h = None

    def bond_dims(self) -> List[int]:
        out = (C.c_int * (self.L + 1))()
        _chk(lib.tt_dmps_bond_dims(self.h, out), "bond_dims")
        return list(out)

    def overlap(self, other=None) -> float:
        """psiphi(self, other) (mps/observables.cpp:382-450); other defaults to self."""
        out = D()
        _chk(lib.tt_dmps_overlap(self.h, (other or self).h, C.byref(out)), "overlap")
        return out.value

    def expectation(self, H, other=None) -> float:
        """psiHphi(self, H, other) (mps/observables.cpp:25-103), unnormalised."""
        out = D()
        _chk(lib.tt_dmps_expectation(self.h, H.h, (other or self).h, C.byref(out)), "expectation")
        return out.value

    def measure_sz(self):
        """(<Sz_i> as an (L,) array, <Sz_i Sz_j> as an (L, L) array), normalised by <psi|psi>."""
        sz = np.zeros(self.L)
        szsz = np.zeros((self.L, self.L))
        _chk(lib.tt_dmps_measure_sz(self.h, sz.ctypes.data_as(PD), szsz.ctypes.data_as(PD)), "measure_sz")
        return sz, szsz


class DMPO:
    """Dense MPO: the hand-written Heisenberg chain, D=5 (models/hams/Heisenberg.cpp:185-208),
    or any spin-1/2 AutoMPO through ``DMPO.from_autompo``."""

    def __init__(self, L: int, dh: Optional[Sequence[float]] = None, tE: float = 0.0, mpo_id: int = 2,
                 _handle=None):
        self.L = L
        self.h = P()
        if _handle is not None:
            self.h = _handle
            return
        arr = (D * L)(*dh) if dh is not None else None
        _chk(lib.tt_dmpo_heisenberg(L, arr, tE, mpo_id, C.byref(self.h)), "dmpo")

    @classmethod
    def from_autompo(cls, ampo: "AutoMPO", N: int, mpo_id: int = 2) -> "DMPO":
        h = P()
        _chk(lib.tt_dmpo_from_autompo(ampo.h, N, mpo_id, C.byref(h)), "dmpo from autompo")
        return cls(N, _handle=h)

    def tensor(self, i: int) -> np.ndarray:
        """Site tensor as an array (left link, ket, bra, right link)."""
        dims = (I64 * 4)()
        _chk(lib.tt_dmpo_tensor(self.h, i, dims, None, 0), "dmpo tensor")
        n = int(np.prod(list(dims)))
        out = np.zeros(n)
        _chk(lib.tt_dmpo_tensor(self.h, i, dims, out.ctypes.data_as(PD), n), "dmpo tensor")
        return out.reshape(list(dims), order="F")

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_dmpo_destroy(self.h)
            self.h = None


def ddmrg_run(psi: DMPS, H: DMPO, nsweeps: int, maxm, cutoff, max_restart):
    """dmrg(MPS&, MPO&, nsweeps, maxm[], cutoff[], max_restart[]) -> (energy, sweep energies, kept per step)."""
    e = D()
    se = (D * max(1, nsweeps))()
    kept = (C.c_int * max(1, 2 * (psi.L - 1) * nsweeps))()
    _chk(lib.tt_ddmrg_run(psi.h, H.h, nsweeps, (C.c_int * len(maxm))(*maxm), len(maxm),
                          (D * len(cutoff))(*cutoff), len(cutoff), (C.c_int * len(max_restart))(*max_restart),
                          len(max_restart), C.byref(e), se, kept), "ddmrg")
    return e.value, list(se)[:nsweeps], list(kept)


class AutoMPO:
    """AutoMPO term accumulator (models/hams/AutoMPO.{h,cpp}); host-side only.

    ``ampo.add(0.5, "S+", i, "S-", j)`` or ``ampo += (0.5, "S+", i, "S-", j)``
    mirrors the reference's ``ampo += 0.5, "S+", i, "S-", j;``."""

    def __init__(self):
        self.h = P()
        _chk(lib.tt_autompo_create(C.byref(self.h)), "autompo create")

    def __del__(self):
        if getattr(self, "h", None):
            lib.tt_autompo_destroy(self.h)
            self.h = None

    def add(self, *args):
        coef, ops, sites, pending = 1.0, [], [], None
        for a in args:
            if isinstance(a, str):
                if pending is not None:
                    raise ValueError("Invalid input to AutoMPO (two strings in a row?)")
                pending = a
            elif pending is not None:
                ops.append(pending.encode())
                sites.append(int(a))
                pending = None
            else:
                coef *= float(a)
        if pending is not None:
            raise ValueError("Invalid input to AutoMPO (missing site number?)")
        if not ops:
            raise ValueError("No operators in HTerm")
        _chk(lib.tt_autompo_add(self.h, coef, len(ops), (C.c_char_p * len(ops))(*ops),
                                (C.c_int * len(sites))(*sites)), "autompo add")
        return self

    def __iadd__(self, term):
        return self.add(*(term if isinstance(term, tuple) else (term,)))

    def __len__(self):
        n = C.c_int()
        _chk(lib.tt_autompo_size(self.h, C.byref(n)), "autompo size")
        return n.value

    def terms(self):
        """[(coef, ((site, op), ...))] in the accumulator's order."""
        out = []
        for k in range(len(self)):
            coef, nops = D(), C.c_int()
            names = C.create_string_buffer(16 * 8)
            sites = (C.c_int * 8)()
            _chk(lib.tt_autompo_term(self.h, k, C.byref(coef), C.byref(nops), names, sites, 8), "autompo term")
            ops = tuple((sites[j], names.raw[16 * j:16 * j + 16].split(b"\0")[0].decode())
                        for j in range(min(nops.value, 8)))
            out.append((coef.value, ops))
        return out

    def link_dims(self, N: int, with_charges: bool = True) -> List[int]:
        dims = (C.c_int * (N + 1))()
        _chk(lib.tt_autompo_link_dims(self.h, N, int(with_charges), dims), "autompo link dims")
        return list(dims)


class LatticeBond(C.Structure):
    _fields_ = [("s1", C.c_int), ("s2", C.c_int), ("type", C.c_int), ("x1", D), ("y1", D), ("x2", D), ("y2", D)]


_proto("tt_lattice", C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(LatticeBond), C.c_int, C.POINTER(C.c_int))
TT_LATTICE_SQUARE, TT_LATTICE_SQUARE_NEXT_NEIGHBOR, TT_LATTICE_TRIANGULAR = 0, 1, 2
TT_LATTICE_SNAKE = 0x100


def _lattice(kind, Nx, Ny, yperiodic):
    n = C.c_int()
    _chk(lib.tt_lattice(kind, Nx, Ny, int(yperiodic), None, 0, C.byref(n)), "lattice")
    buf = (LatticeBond * max(1, n.value))()
    _chk(lib.tt_lattice(kind, Nx, Ny, int(yperiodic), buf, n.value, C.byref(n)), "lattice")
    return [(b.s1, b.s2, b.type, b.x1, b.y1, b.x2, b.y2) for b in buf[:n.value]]


def square_lattice(Nx: int, Ny: int, yperiodic: bool = False, snake: bool = False):
    """squareLattice (models/lattice/square.h:25-58): (s1, s2, type, x1, y1, x2, y2), 1-based sites.
    snake=True numbers the sites in snake order (odd columns upward, even columns downward)."""
    return _lattice(TT_LATTICE_SQUARE | (TT_LATTICE_SNAKE if snake else 0), Nx, Ny, yperiodic)


def square_next_neighbor(Nx: int, Ny: int, yperiodic: bool = False, snake: bool = False):
    """squareNextNeighbor (models/lattice/square.h:60-103); type 1 nearest, 2 next nearest.
    snake=True numbers the sites in snake order (odd columns upward, even columns downward)."""
    return _lattice(TT_LATTICE_SQUARE_NEXT_NEIGHBOR | (TT_LATTICE_SNAKE if snake else 0), Nx, Ny, yperiodic)


def triangular_lattice(Nx: int, Ny: int, yperiodic: bool = True):
    """triangularLattice (models/lattice/triangular.h:25-64)."""
    return _lattice(TT_LATTICE_TRIANGULAR, Nx, Ny, yperiodic)


def set_precision(op: str = "fp64", heff: str = "fp64", env: str = "fp64"):
    """Contraction precisions on this thread ("fp64", "tf32", "tf32x3",
    "tf32-auto", "tf32x3-auto"): op for QTensor/dense contractions, heff for
    the Davidson H_eff*x products, env for the environment updates.  The mixed
    form of the DMRG sweep is set_precision(heff="tf32x3-auto",
    env="tf32x3-auto"): 3xTF32 on the tensor cores for the contractions the
    cost model predicts faster there, FP64 for the rest."""
    _chk(lib.tt_dmrg_set_precision(PRECISIONS[op], PRECISIONS[heff], PRECISIONS[env]), "set_precision")


def set_davidson_control(device: bool = True):
    """tensor_davidsonIT control on the device (one synchronisation per call,
    host loop on Gram-Schmidt failure) or on the host (reads back every iteration)."""
    _chk(lib.tt_dmrg_set_davidson(int(device)), "set_davidson")


def heff_parts() -> dict:
    """Totals over this thread's device-resident Davidson products: device ms
    and algorithmic flops of L*x, *mid, *R, and the *mid contractions'
    algorithmic bytes."""
    ms, fl, mb = (D * 3)(), (D * 3)(), D()
    _chk(lib.tt_dmrg_heff_parts(ms, fl, C.byref(mb)), "heff_parts")
    return {"ms": list(ms), "flops": list(fl), "mid_bytes": mb.value}


def eig_redo_count(ctx) -> int:
    """Eigenproblems whose vectors were recomputed by the cluster kernel after
    CholeskyQR2 found a collapsed inverse-iteration vector (device-wide)."""
    n = I64()
    _chk(lib.tt_eig_redo_count(ctx.h, C.byref(n)), "eig_redo_count")
    return n.value


def planning_counters() -> dict:
    """Host time spent on contraction structures and plans (this thread):
    seconds and counts since the thread started."""
    ts, tp = D(), D()
    ns, np_ = I64(), I64()
    _chk(lib.tt_dmrg_planning_counters(C.byref(ts), C.byref(ns), C.byref(tp), C.byref(np_)), "planning_counters")
    return {"structure_s": ts.value, "structures": ns.value, "plan_s": tp.value, "plans": np_.value}


def plan_timers() -> list:
    """Host seconds of the contraction planner's stages on this thread: pair
    tables, precision choice, tile tasks / chunks, packing jobs, uploads."""
    out = (D * 5)()
    _chk(lib.tt_contract_plan_timers(out, 5), "plan timers")
    return list(out)


def cache_stats() -> dict:
    """This thread's contraction cache: entries, plan device bytes, evictions."""
    e, b, r, n = I64(), I64(), I64(), I64()
    _chk(lib.tt_dmrg_cache_stats(C.byref(e), C.byref(b), C.byref(r), C.byref(n)), "cache_stats")
    return {"entries": e.value, "plan_bytes": b.value, "evictions": r.value, "evicted": n.value}


def davidson_refills() -> int:
    """Gram-Schmidt failures refilled inside the device-resident loop (this thread)."""
    n = I64()
    _chk(lib.tt_dmrg_davidson_refills(C.byref(n)), "davidson_refills")
    return n.value


def davidson_fallbacks() -> int:
    n = I64()
    _chk(lib.tt_dmrg_davidson_fallbacks(C.byref(n)), "davidson_fallbacks")
    return n.value
