"""The synthetic workloads' shapes and the run_case partitions (host logic, CPU).

Each workload must fit the library's limits: subdomains with ny*nz <= 256
lines and at most 8192 cells, at most 4096 coarse unknowns per virtual rank
(subdomains per rank x en_lv1) and 8192 level-3 unknowns.
"""
import numpy as np
import pytest

from premixfem_b200 import fields
from premixfem_b200.run_case import make_case
from premixfem_b200.solver import options_string


def _check_partition(mesh, sd_per_rank, vranks, k, en2=4):
    total = [a * b for a, b in zip(sd_per_rank, vranks)]
    sub = [-(-m // t) for m, t in zip(mesh, total)]  # largest subdomain per axis (near-equal split)
    assert sub[1] * sub[2] <= 256 and np.prod(sub) <= 8192, sub
    assert np.prod(sd_per_rank) * k <= 4096
    assert np.prod(vranks) * en2 <= 8192
    return sub


def test_layered_workload_partition():
    prob, opts = make_case("layered", 0, 2)
    assert prob["mesh"] == (60, 220, 85) and prob["dom"] == (1200.0, 2200.0, 170.0)
    assert not prob["dirichlet"] and abs(prob["source"].sum()) < 1e-12
    sub = _check_partition(prob["mesh"], opts["pmf_sd"], opts["pmf_vranks"], opts["en_lv1"])
    assert sub == [10, 10, 5]
    assert "-ksp_constant_null_space" in options_string(opts)
    k = prob["kappa"][0]
    assert k[40:].max() / k[40:].min() == pytest.approx(1e6)


def test_large_workload_partition_scaled():
    prob, opts = make_case("large", 256, 5)
    assert prob["mesh"] == (256, 256, 128) and prob["dirichlet"] == {"z-": 0.0}
    sd = (opts["sd"],) * 3
    sub = _check_partition(prob["mesh"], sd, opts["pmf_vranks"], opts["en_lv1"])
    assert sub == [16, 16, 16]


def test_problem_batch_statistics():
    batch = fields.grf_batch(count=64, seed=3)
    assert len(batch) == 64
    sizes = np.array([p["mesh"] for p, _ in batch])
    assert sizes.min() >= 24 and sizes.max() <= 80
    assert 7.0e6 < np.prod(sizes, axis=1).sum() < 11.0e6  # E[N] = 52^3 x 64 ~ 9.0 M cells
    for p, srcs in batch:
        assert len(srcs) == 4 and p["dirichlet"] == {"x+": 0.0}
        assert np.allclose(srcs[0], srcs[0].flat[0])  # the unit source
        t = fields.tiles(p["mesh"])
        _check_partition(p["mesh"], t, (1, 1, 1), 4)
        assert all(-(-m // s) <= 8 for m, s in zip(p["mesh"], t))
