"""GPU: failures made on the host, and the library's recovery from them.

Device allocations fail on demand through pepcg_debug_fail_allocations (a
host-side injection: the allocation call is answered with an error before it
reaches the device).  A grow or traverse that meets the failure must return
PEPCG_ERR_OOM with a message, leave no tree behind, and the same context must
then work again and give the results of a fresh context."""
import numpy as np
import pytest

import pepc_b200 as P
from tests.datasets import cube

pytestmark = pytest.mark.gpu


@pytest.fixture
def no_injection(gpu):
    yield
    P.lib().pepcg_debug_fail_allocations(-1)


@pytest.mark.parametrize("after", [0, 1, 5, 12, 20])
def test_grow_allocation_failure_then_recovery(no_injection, after):
    x, y, z, q = cube(30000, 81, charges="normal")
    ref = P.TreeCode(theta2=0.25, eps2=1e-4)
    g_ref = ref.pepc_grow_tree(x, y, z, q)
    r_ref = ref.pepc_traverse_tree(g_ref.x, g_ref.y, g_ref.z, keys=g_ref.key)
    ref.close()
    tc = P.TreeCode(theta2=0.25, eps2=1e-4)
    P.lib().pepcg_debug_fail_allocations(after)
    with pytest.raises(P.PepcgError) as e:
        tc.pepc_grow_tree(x, y, z, q)
    assert e.value.code == P.PEPCG_ERR_OOM
    assert "injected" in str(e.value)
    P.lib().pepcg_debug_fail_allocations(-1)
    # nothing was grown: a traverse is refused, not run on stale data
    with pytest.raises(P.PepcgError) as e2:
        tc.pepc_traverse_tree(x[:10], y[:10], z[:10])
    assert e2.value.code == P.PEPCG_ERR_NO_TREE
    g = tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    assert np.array_equal(g.perm, g_ref.perm)
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], r_ref[k]), k
    tc.close()


def test_traverse_allocation_failure_keeps_the_tree(no_injection):
    x, y, z, q = cube(20000, 82, charges="normal")
    tc = P.TreeCode(theta2=0.25, eps2=1e-4)
    g = tc.pepc_grow_tree(x, y, z, q)
    P.lib().pepcg_debug_fail_allocations(0)
    with pytest.raises(P.PepcgError) as e:
        # foreign targets need staging buffers the grow did not allocate
        tc.pepc_traverse_tree(np.linspace(0, 1, 70000), np.full(70000, 0.5), np.full(70000, 0.5))
    assert e.value.code == P.PEPCG_ERR_OOM
    P.lib().pepcg_debug_fail_allocations(-1)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    assert np.all(np.isfinite(r["pot"])) and np.all(r["work"] > 0)
    tc.close()
