"""The autotuner's block sizes (128, 256 or 512 threads per fused block).

mpc_prepare measures a request's kind (family, sampler, step bucket) at the
three block sizes and keeps the fastest; mpc_price then uses it.  A block
size changes only the tile partition and the order of the in-block sums, so
every forced shape gives the autotuned price to 1e-12 relative.
"""

import pytest

from montepath_b200.requests import make_request

pytestmark = pytest.mark.gpu

KINDS = [
    ("european_call", dict(model="heston", n_paths=1 << 18, n_steps=64, seed=8, sampling="scrambled_sobol",
                           kappa=2.0, vol_of_vol=0.5, rho=-0.7)),
    ("european_call", dict(method="stepwise", n_paths=300_000, n_steps=64, seed=9, sampling="counter_hash")),
    ("arithmetic_asian_call", dict(n_paths=200_000, n_steps=48, seed=10, sampling="scrambled_sobol",
                                   technique="antithetic")),
    ("basket_call", dict(method="stepwise", n_steps=16, n_paths=100_000, seed=11, sampling="counter_hash",
                         spots=[100, 95, 105, 98, 102], sigmas=[0.2, 0.25, 0.3, 0.15, 0.22], weights=[0.2] * 5,
                         corr=0.3, k=100)),
]


@pytest.mark.parametrize("workload,kw", KINDS)
def test_prepare_tunes_block_and_forced_shapes_agree(backend, workload, kw):
    r = make_request(workload, kw)
    art = backend.prepare(r)
    assert art.block_size in (128, 256, 512)
    tuned = backend.price(r)
    for block in (128, 256, 512):
        forced = backend.price(make_request(workload, dict(kw, block_size=block)))
        assert abs(forced.price - tuned.price) <= 1e-12 * abs(tuned.price), (block, forced.price, tuned.price)
        assert abs(forced.stderr - tuned.stderr) <= 1e-9 * tuned.stderr
        art_b = backend.prepare(make_request(workload, dict(kw, block_size=block)))
        assert art_b.block_size == block
        assert art_b.tiles * block * art_b.paths_per_thread >= (r.n_paths + 1) // 2


def test_block_choice_is_stable(backend):
    """A kind is measured once per context: preparing it again returns the same block."""

    r = make_request(*KINDS[0][:1], KINDS[0][1])
    first = backend.prepare(r).block_size
    for _ in range(3):
        assert backend.prepare(r).block_size == first
