"""The timeout path of the tensor-core contraction kernel.

Every mbarrier wait of the persistent tcgen05 kernel is bounded.  With the
context's main-loop limit lowered to 0 polls (tt_ctx_set_wait_limit), the
first wait of every CTA gives up at once, exactly as a wait on a flag that
nothing sets would after its limit: the kernel records TT_ERR_TIMEOUT, lets
the bulk copies it issued land (with the full limit), frees its tensor memory
and returns.  The host must then refuse to read results -- every
synchronisation of the context returns TT_ERR_TIMEOUT -- and, once the status
is cleared and the limit restored, the same context must contract correctly.
No GPU is faulted or hung: the kernel returns by itself.
"""
import numpy as np
import pytest

from oracle.qtensor import QIndex, QTensor, Inward, Outward, Link, contract, qn, to_dense

pytestmark = pytest.mark.gpu


def _index(arrow, name, sectors, level=0):
    ix = QIndex(arrow, name, Link, level)
    for q, d in sectors:
        ix.add_qn(qn(q), d)
    return ix


def test_tensor_core_timeout_is_reported_and_the_context_recovers():
    import tt_b200
    rng = np.random.default_rng(5)
    i = _index(Inward, "i", [(-2, 150), (0, 300), (2, 90)])
    k = _index(Outward, "k", [(-2, 70), (0, 260), (2, 130)])
    j = _index(Inward, "j", [(-2, 40), (0, 280), (2, 200)])
    A = QTensor([i, k])
    A.init_block()
    B = QTensor([k.dagged(), j])
    B.init_block()
    for T in (A, B):
        for b in T.blocks:
            b[...] = rng.standard_normal(b.shape)
    want = to_dense(contract(A, B))
    ctx = tt_b200.Context(0)
    try:
        gA, gB = tt_b200.QTensor.from_oracle(A), tt_b200.QTensor.from_oracle(B)
        tt_b200.set_precision(op="tf32x3")
        assert ctx.device_status() == tt_b200.TT_OK
        ctx.set_wait_limit(0)
        C = gA * gB
        with pytest.raises(tt_b200.TTError, match="status %d" % tt_b200.TT_ERR_TIMEOUT):
            C.to_oracle()  # the read synchronises and finds the timed-out contraction
        assert ctx.device_status() == tt_b200.TT_ERR_TIMEOUT
        with pytest.raises(tt_b200.TTError):
            ctx.sync()  # sticky until cleared
        ctx.set_wait_limit(-1)
        ctx.clear_device_status()
        assert ctx.device_status() == tt_b200.TT_OK
        for _ in range(2):  # the same cached plan, now with the full limit
            got = to_dense((gA * gB).to_oracle())
            assert np.linalg.norm(got - want) / np.linalg.norm(want) < 2e-6
        assert ctx.device_status() == tt_b200.TT_OK
        del C, gA, gB
    finally:
        tt_b200.set_precision()
        ctx.set_wait_limit(-1)
        ctx.close()
