"""The entry point's smoke(): SpMV and Jacobi-PCG on a small grid,
bit-identical to the oracle."""
import pytest

pytestmark = pytest.mark.gpu


def test_smoke_entry_point(gpu):
    import __graft_entry__
    __graft_entry__.smoke()
