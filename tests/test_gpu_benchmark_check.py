"""GPU: pepc-benchmark's own correctness run (benchmark/benchmark.xml, tag check;
frontends/pepc-benchmark/pepc.f90 and module_helper.f90) on the device time loop
-- the reference's acceptance criterion for a whole simulation, not a per-particle
comparison.

A Kaplan Coulomb explosion of n electrons (q = -2/n, m = 1e-3), theta2 = 0.25,
eps2 = 1e-4, dt = 0.02, run to the check step sqrt(n / 1000) * 210, where the
velocity histogram of the particles at radii 7 .. 8.5 must show exactly two
peaks (test_histogram: runs of occupied bins).  The accelerations scale as 1/n
and the check step as sqrt(n), so the state there is the same for any n; the
test runs n = 65,536 (1,800 steps), `bench.py --workload benchmark-check` the
reference's 1,048,576 (6,900 steps).  Also checked: the total energy's drop
over the run (the JUBE pattern egy_drop; the reference sets no bound, 2 % is
this test's), the direct-sum L2 error (relative 1e-3), and that the mixed and
plain forms end in the same histogram and energy (to 1e-4)."""
import numpy as np
import pytest
import torch

import pepc_b200 as P
from bench import benchmark_check

pytestmark = pytest.mark.gpu


def test_pepc_benchmark_check(gpu):
    dev = torch.device("cuda", 0)
    res = {}
    for name, prec, walk in (("mixed", P.PRECISION_MIXED, P.WALK_GROUP),
                             ("plain", P.PRECISION_PLAIN, P.WALK_PER_TARGET)):
        r = benchmark_check(P, torch, dev, 65536, prec, walk)
        print(name, {k: v for k, v in r.items() if k != "histogram"})
        assert r["check_step"] == 1800
        assert r["histogram_peaks"] == 2, r["histogram"]
        assert r["egy_drop_pct"] < 2.0
        assert r["l2_rel_max"] < 1e-3
        res[name] = r
    hm, hp = np.array(res["mixed"]["histogram"]), np.array(res["plain"]["histogram"])
    assert np.abs(hm - hp).sum() <= 1e-3 * hp.sum()
    assert abs(res["mixed"]["energy_last"] - res["plain"]["energy_last"]) <= \
        1e-4 * abs(res["plain"]["energy_last"])
