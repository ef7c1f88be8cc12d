"""The INT8 tensor-core kernel's give-up path, made to run on purpose without
faulting or hanging the GPU.

Every pipeline wait of the tcgen05 kernels is bounded.  With the failure-test
settings read at context creation (BW_TEST_WAIT_LIMIT: tries per wait;
BW_TEST_HOLD_FIRST_STAGE: CTA 0 never fills its first stage), the MMA thread's
wait for that stage runs out: the CTA raises its give-up flag, every role winds
down, in-flight copies and MMAs drain, TMEM is freed and the kernel returns.
The host must report status 2 with the wait's name, and a fresh context on the
same device must still match the oracle.
"""
import numpy as np
import pytest

import oracle
from prym_green_ancillary_b200 import EngineError, KoszulEngine

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPE = (8, 4, 6, 5, 32003, 16, 16)   # r, k, dim_in, dim_out, p, n, m


def _forward(eng, Y, shape, dev):
    y = torch.from_numpy(Y.view(np.int32)).to(dev)
    z = torch.empty((shape.n_tgt, shape.nb), dtype=torch.int32, device=dev)
    eng.forward(y, z)
    torch.cuda.synchronize()
    return z.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("producer", ["cpasync8", "cpasync16", "hybrid"])
def test_wait_that_runs_out_returns_status_2_and_context_stays_usable(producer, monkeypatch):
    """Every stage producer: the cp.async warps alone (8 or 16 of them), and
    TMA gathers beside them."""
    shape = oracle.KoszulShape(*SHAPE)
    maps, diag, X, Y = oracle.seeded_problem(shape, 41)
    dev = torch.device("cuda", 0)
    if producer.startswith("cpasync"):
        monkeypatch.setenv("BW_I8_PRODUCER_WARPS", producer[len("cpasync"):])
        producer = "cpasync"
    monkeypatch.setenv("BW_I8_PRODUCER", producer)
    monkeypatch.setenv("BW_TEST_WAIT_LIMIT", "100000")
    monkeypatch.setenv("BW_TEST_HOLD_FIRST_STAGE", "1")
    with KoszulEngine(*SHAPE, maps=maps, diag=diag, form="int8") as eng:
        assert ("hybrid" in eng.plan) == (producer == "hybrid")
        with pytest.raises(EngineError) as err:
            _forward(eng, Y, shape, dev)
        assert err.value.status == 2
        assert "gave up waiting (ERR_WAIT_" in str(err.value)
    monkeypatch.delenv("BW_TEST_WAIT_LIMIT")
    monkeypatch.delenv("BW_TEST_HOLD_FIRST_STAGE")
    monkeypatch.delenv("BW_I8_PRODUCER_WARPS", raising=False)
    # the CUDA context is intact: a fresh engine on the same device is exact
    with KoszulEngine(*SHAPE, maps=maps, diag=diag, form="int8") as eng:
        np.testing.assert_array_equal(_forward(eng, Y, shape, dev), oracle.forward(shape, maps, Y))
        seq, yf = eng.sequence_host(X, Y, 9)
    want, yf_want = oracle.sequence(shape, maps, diag, X, Y, 9)
    np.testing.assert_array_equal(seq, want)
    np.testing.assert_array_equal(yf, yf_want)
