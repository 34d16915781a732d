"""The time-out path of the tensor-core kernels' bounded device waits,
exercised without faulting or hanging the GPU: emc_wait_probe runs one wait
on an mbarrier that nothing completes, with a 2 ms limit, through the same
wait routine the contractions use.  The call must report EMC_ERR_TIMEOUT
with the wait site, and the context must then iterate exactly as a fresh
one does."""
import numpy as np
import pytest

from parity import make_ctx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["mixed", "fp32"])
def test_bounded_wait_gives_up_and_context_stays_usable(prec):
    import emc_b200 as E
    from emc_b200 import workloads as W
    d = W.make("tiny16")
    with make_ctx(d, "poisson", "nearest", prec) as ref:
        ref.iterate()
        m_ref = ref.get_model()
    with make_ctx(d, "poisson", "nearest", prec) as ctx:
        with pytest.raises(E.EmcError) as ei:
            ctx.wait_probe(2000)
        assert ei.value.status == 4  # EMC_ERR_TIMEOUT
        assert "wait 90" in str(ei.value)
        ctx.synchronize()  # the status word was cleared
        ctx.iterate()
        np.testing.assert_allclose(ctx.get_model(), m_ref, rtol=1e-6, atol=1e-7)


def test_wait_probe_rejects_bad_limits():
    import emc_b200 as E
    from emc_b200 import workloads as W
    with make_ctx(W.make("tiny16")) as ctx:
        for bad in (0, 2_000_000):
            with pytest.raises(E.EmcError) as ei:
                ctx.wait_probe(bad)
            assert ei.value.status == 1
