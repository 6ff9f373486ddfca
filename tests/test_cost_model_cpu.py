"""The cost model behind the automatic mixed precision (TT_PREC_TF32X3_AUTO),
evaluated on the host through tt_contract_predict (no device needed).

Pins the choices measured on B200 for the J1-J2 cylinder at bond dimension
1024: the contraction of (L x) with the two-site MPO (k = n = 14, bandwidth
bound) stays FP64 (measured 354 us FP64 against 685 us on the tensor cores
with packing), while L*x-shaped contractions (m ~ 1400, n ~ k ~ 100) go to
the tensor cores (measured 141 against 301 us), as does one 2048^3 block;
tiny contractions, dominated by the extra launches, stay FP64.
"""
import ctypes as C

import pytest

MAXM = 6
TT_PREC_FP64, TT_PREC_TF32X3, TT_PREC_TF32X3_AUTO = 0, 2, 4


class OutBlock(C.Structure):
    _fields_ = [("c_off", C.c_int64), ("m", C.c_int32), ("n", C.c_int32), ("ldc", C.c_int32)]


class BlockPair(C.Structure):
    _fields_ = [("out_block", C.c_int32), ("n_m", C.c_int32), ("n_k", C.c_int32), ("n_n", C.c_int32),
                ("a_off", C.c_int64), ("b_off", C.c_int64),
                ("m_dims", C.c_int32 * MAXM), ("k_dims", C.c_int32 * MAXM), ("n_dims", C.c_int32 * MAXM),
                ("a_m_stride", C.c_int64 * MAXM), ("a_k_stride", C.c_int64 * MAXM),
                ("b_k_stride", C.c_int64 * MAXM), ("b_n_stride", C.c_int64 * MAXM)]


def _lib():
    import tt_b200
    f = tt_b200.lib.tt_contract_predict
    f.restype = C.c_int
    f.argtypes = [C.POINTER(OutBlock), C.c_int, C.POINTER(BlockPair), C.c_int, C.c_int, C.c_int,
                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    return tt_b200, f


def _contraction(blocks):
    """blocks: list of (m, n, [k of each pair]); every pair has its own A and B block."""
    outs, pairs = [], []
    c_off = a_off = b_off = 0
    for o, (m, n, ks) in enumerate(blocks):
        outs.append(OutBlock(c_off, m, n, m))
        c_off += m * n
        for k in ks:
            p = BlockPair()
            p.out_block, p.n_m, p.n_k, p.n_n = o, 1, 1, 1
            p.a_off, p.b_off = a_off, b_off
            p.m_dims[0], p.k_dims[0], p.n_dims[0] = m, k, n
            p.a_m_stride[0], p.a_k_stride[0] = 1, m
            p.b_k_stride[0], p.b_n_stride[0] = 1, k
            pairs.append(p)
            a_off += m * k
            b_off += k * n
    return (OutBlock * len(outs))(*outs), len(outs), (BlockPair * len(pairs))(*pairs), len(pairs)


def _predict(blocks, num_sms=148):
    tt_b200, f = _lib()
    o, no, p, npairs = _contraction(blocks)
    a, b, ch = C.c_double(), C.c_double(), C.c_int()
    rc = f(o, no, p, npairs, TT_PREC_TF32X3_AUTO, num_sms, C.byref(a), C.byref(b), C.byref(ch))
    assert rc == 0, tt_b200.lib.tt_get_last_error()
    assert a.value > 0 and b.value > 0
    return a.value, b.value, ch.value


def test_bandwidth_bound_mpo_contraction_stays_fp64():
    # (L x) * (W1 W2) over (w, s1, s2): m = a' b ~ 10^4, n = k = 14, four pairs per output block
    us64, ustc, choice = _predict([(100 * 100, 14, [14, 14, 14, 14])] * 60)
    assert choice == TT_PREC_FP64, (us64, ustc)


def test_compute_bound_environment_contractions_go_to_tensor_cores():
    # L * x over a: m = a' w ~ 1400, n = b ~ 100, k = a ~ 100
    us64, ustc, choice = _predict([(1400, 100, [100])] * 90)
    assert choice == TT_PREC_TF32X3, (us64, ustc)
    assert ustc < 0.8 * us64


def test_large_block_goes_to_tensor_cores_and_tiny_one_stays_fp64():
    us64, ustc, choice = _predict([(2048, 2048, [2048])])
    assert choice == TT_PREC_TF32X3 and ustc < 0.25 * us64, (us64, ustc)
    _, _, tiny = _predict([(2, 2, [2, 4])] * 3)
    assert tiny == TT_PREC_FP64


def test_rejects_forced_precisions_and_bad_pairs():
    tt_b200, f = _lib()
    o, no, p, npairs = _contraction([(8, 8, [8])])
    a, b, ch = C.c_double(), C.c_double(), C.c_int()
    assert f(o, no, p, npairs, TT_PREC_TF32X3, 148, C.byref(a), C.byref(b), C.byref(ch)) != 0
    p[0].out_block = 5
    assert f(o, no, p, npairs, TT_PREC_TF32X3_AUTO, 148, C.byref(a), C.byref(b), C.byref(ch)) != 0
