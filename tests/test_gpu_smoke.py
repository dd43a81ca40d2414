"""The build entry's smoke check (a small forward and backward selection on
cuda:0, each compared bit for bit with the CPU oracle) runs with the GPU suite."""
import pytest

pytestmark = pytest.mark.gpu


def test_smoke_entry_point():
    import __graft_entry__

    __graft_entry__.smoke()
