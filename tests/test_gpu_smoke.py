"""The build entry point's smoke check (one small level call of the batched FP32 path and of the
reference-stream path, each against the oracle on the same streams) runs inside the GPU suite, so
a change that breaks it shows up with the other GPU tests."""
import pytest

pytestmark = pytest.mark.gpu


def test_graft_entry_smoke(nm):
    import __graft_entry__
    __graft_entry__.smoke()
