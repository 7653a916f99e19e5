"""Free-running integration of the 2->4 multichannel workload on both sides,
nothing copied between them: the CUDA library (on-device Philox uniforms,
seed 7) and the reference's own MultiChannel (oracle/_ref, its MPI mode over
host processes, MultiChannel.hh:184-212) each run 20 adapting iterations of
1e6 accepted points from uniform grids and equal channel weights.  The
pooled integrals (MultiChannel.cc:69-77: the sums over all iterations) must
agree within 3 sigma of the combined statistical error.

Each side's error against a high-statistics FP64 estimate is stated too:
the GPU continues from its adapted grids with 100 non-adapting iterations of
1e6 points (a 1e8-point estimate, ~10x smaller error than either run), and
each side's pull against it is printed and bounded.

The reference's speed on the host sets the size: 1e6 points per iteration
split over the ranks (ncalls / size each, MultiChannel.hh:209) when the host
has at least 16 cores; with fewer, 62,500 points per rank and iteration
(the test prints the size it ran).
"""
import os

import numpy as np
import pytest

from chili_b200 import abi, channels, gpu, workloads

pytestmark = pytest.mark.gpu

ITERATIONS = 20
SEED = 7


def _cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _pooled_mean_error(rows):
    pooled = np.zeros(6)
    for r in rows:
        pooled += np.array(r) * np.array([1, 0, 0, 1, 1, 1])
    return gpu.stats_mean_error(pooled)


def test_free_running_integral_agrees_with_the_reference(ctx_factory):
    from oracle import ref
    from oracle.mpi_ranks import RefMPI
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    nranks = min(_cores(), 32)
    ncalls = 1_000_000 if nranks >= 16 else 62_500 * nranks
    with RefMPI(nranks, n_out=4, bins=100, ncalls=ncalls, fkind="PROPAGATOR", seed=SEED, cuts=True) as M:
        ref_rows = []
        ref_seconds = 0.0
        for _ in range(ITERATIONS):
            st, _, _, sec = M.iterate()
            ref_rows.append(st)
            ref_seconds += sec
        a_r, _, _, _ = M.state(0)
    ncalls_ref = M.ncalls_rank * nranks

    cs = workloads.channel_set(4)
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, 100)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess_cuts(cs.sqrts)
    params = workloads.mc_params(ncalls_ref, iterations=ITERATIONS)
    rows, counter = [], 0
    for _ in range(ITERATIONS):
        st, info = ctx.multichannel_iterate(params, seed=SEED, counter=counter, guard=True)
        counter += info.points_tried
        rows.append(st.as_tuple())
    a_g = ctx.get_alpha()[0]

    m_g, e_g = _pooled_mean_error(rows)
    m_r, e_r = _pooled_mean_error(ref_rows)
    pull = (m_g - m_r) / np.hypot(e_g, e_r)

    # the high-statistics estimate on the GPU's adapted grids
    fixed = workloads.mc_params(1_000_000, iterations=100, should_optimize=0)
    hi = []
    for k in range(100):
        st, info = ctx.multichannel_iterate(fixed, seed=SEED + 1, counter=counter, guard=True)
        counter += info.points_tried
        hi.append(st.as_tuple())
    m_h, e_h = _pooled_mean_error(hi)
    print(f"\nfree-running 2->4, {ITERATIONS} x {ncalls_ref} points ({nranks} reference ranks, "
          f"{ref_seconds:.1f} s): GPU {m_g:.6e} +- {e_g:.2e} ({e_g / m_g:.2e}), reference {m_r:.6e} +- {e_r:.2e} "
          f"({e_r / m_r:.2e}), pull {pull:+.2f}; 1e8-point estimate {m_h:.6e} +- {e_h:.2e}: GPU "
          f"{(m_g - m_h) / m_h:+.2e} ({(m_g - m_h) / np.hypot(e_g, e_h):+.2f} sigma), reference "
          f"{(m_r - m_h) / m_h:+.2e} ({(m_r - m_h) / np.hypot(e_r, e_h):+.2f} sigma)")
    assert abs(pull) < 3.0, (m_g, e_g, m_r, e_r)
    assert abs(m_g - m_h) < 4.0 * np.hypot(e_g, e_h)
    assert abs(m_r - m_h) < 4.0 * np.hypot(e_r, e_h)
    # both adapted the channel weights to the same shape (the statistics of
    # 2e7 points each): the largest weights sit on the same channels
    assert set(np.argsort(a_g)[-3:]) & set(np.argsort(a_r)[-3:])
