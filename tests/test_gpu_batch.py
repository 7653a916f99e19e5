"""Batched integrands (chili_gpu_batch_*): every task of one persistent,
graph-replayed launch against the oracle run alone on the same
counter-based uniforms (task k: Philox key seed + k, counters
(iteration << 32) + point).

Camel tasks follow Vegas::operator() + AdaptiveMap::Adapt
(Vegas.cc:18-52); multichannel tasks follow MultiChannel::operator() +
Train (MultiChannel.hh:182-251) with its retry loop (points drawn until
ncalls of them pass PreProcess with a finite value; option batch_retry 1),
or with a fixed budget of ncalls drawn points (option batch_retry 0, the
default; the oracle's set_fixed_budget).  Bars: counts and finite counts exact,
sums within 1e-11 relative on the first iteration (CUDA's and the C
library's exp and log differ by an ulp), 1e-9 on later ones (the
histograms are summed with atomics, so later iterations run on grids that
agree to rounding only)."""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from oracle import port

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.where(a == b, 0.0, d)


def camel_task(rng, dims, ncalls, bins):
    sigma = rng.uniform(0.05, 0.2)
    a, b = rng.uniform(0.2, 0.8, dims), rng.uniform(0.2, 0.8, dims)
    return {"kind": "camel", "dims": dims, "bins": bins, "ncalls": ncalls, "grid_alpha": 1.5,
            "params": workloads.camel_params(dims, sigma, a, b)}


def mc_task(n_out, sqrts, ncalls, bins, cuts=False):
    t = {"kind": "multichannel", "channels": workloads.channel_set(n_out, sqrts), "bins": bins,
         "ncalls": ncalls, "grid_alpha": 1.0, "beta": 0.25, "min_alpha": 1e-5,
         "fkind": abi.CHILI_FUNC_PROPAGATOR, "params": channels.propagator_params(),
         "pre": abi.CHILI_PRE_FINITE}
    if cuts:
        t["pre"] = abi.CHILI_PRE_CUTS
        t["pre_cuts"] = (sqrts, 30.0, 99.0, 0.4)
    return t


def oracle_camel(t, seed, iterations):
    edges = np.tile(np.linspace(0.0, 1.0, t["bins"] + 1), (t["dims"], 1))
    out = []
    for it in range(iterations):
        u = port.philox_uniforms(seed, it << 32, t["ncalls"], t["dims"])
        st, _, edges = port.vegas_iterate(edges, t["grid_alpha"], t["params"], u, adapt=True)
        out.append((st.as_tuple(), edges.copy(), None))
    return out


def oracle_mc(t, seed, iterations, retry=True):
    """The oracle on the task's uniforms (Philox key seed, counters
    (iteration << 32) + point): with the retry loop it consumes rows until
    ncalls points are accepted, with a fixed budget exactly ncalls rows."""
    cs = t["channels"]
    params = workloads.mc_params(t["ncalls"], beta=t["beta"], min_alpha=t["min_alpha"],
                                 grid_alpha=t["grid_alpha"])
    O = port.MultiChannel(cs, t["bins"], params, t["fkind"], t["params"], pre=abi.CHILI_PRE_FINITE)
    if t["pre"] == abi.CHILI_PRE_CUTS:
        O.set_cuts(*t["pre_cuts"])
    O.set_fixed_budget(not retry)
    rows = 16 * t["ncalls"] + 4096 if retry else t["ncalls"]
    out = []
    for it in range(iterations):
        u = port.philox_uniforms(seed, it << 32, rows, cs.ndims + 1)
        st, info = O.iterate(u)
        if retry:
            assert info.points_tried >= t["ncalls"] and st.n == info.points_tried
        else:
            assert info.points_tried == t["ncalls"]
        out.append((st.as_tuple(), O.get_grids(), O.get_alpha()[0]))
    return out


def check_task(k, st_gpu, edges, alpha, want, it):
    st_o, e_o, a_o = want
    n, mn, mx, s, s2, nf = st_gpu
    assert n == st_o[0] and nf == st_o[5], (k, it)
    tol = 1e-11 if it == 0 else 1e-9
    assert rel(mn, st_o[1]) < tol and rel(mx, st_o[2]) < tol, (k, it)
    assert rel(s, st_o[3]) < tol and rel(s2, st_o[4]) < tol, (k, it)
    assert np.max(rel(edges.reshape(e_o.shape), e_o)) < 1e3 * tol, (k, it)
    if a_o is not None:
        assert np.max(rel(alpha, a_o)) < 1e3 * tol, (k, it)


def run_and_check(ctx, tasks, seed, iterations, retry=True):
    ctx.batch_set(tasks)
    want = [oracle_camel(t, seed + k, iterations) if t["kind"] == "camel" else
            oracle_mc(t, seed + k, iterations, retry=retry) for k, t in enumerate(tasks)]
    stats = []
    grids = []
    infos = []
    for it in range(iterations):
        st, info = ctx.batch_iterate(1, seed=seed, adapt=True)
        stats.append(st[0])
        infos.append((info.retry_rounds, info.ms_per_iteration))
        grids.append([ctx.batch_get_grid(k) for k in range(len(tasks))])
    for it in range(iterations):
        for k in range(len(tasks)):
            e, a = grids[it][k]
            check_task(k, stats[it][k], e, a, want[k][it], it)
    return info, infos


def test_camel_tasks_match_the_oracle(ctx_factory):
    rng = np.random.default_rng(3)
    tasks = [camel_task(rng, 2, 3000, 20), camel_task(rng, 5, 70001, 50), camel_task(rng, 9, 12345, 30),
             camel_task(rng, 12, 1, 40)]
    info, _ = run_and_check(ctx_factory(), tasks, seed=5, iterations=3)
    assert info.points == sum(t["ncalls"] for t in tasks)
    assert info.block in (128, 256) and info.points_per_thread in (1, 2, 4)


@pytest.mark.parametrize("mode", ["grouped", "grouped_small_waves", "grouped_fixed", "grouped_fixed_small_waves",
                                  "task_chains", "one_kernel"])
def test_multichannel_tasks_match_the_oracle(ctx_factory, mode):
    """Every weight pass of the batched multichannel tasks: the phased pass
    in waves of pieces, one launch per step and wave (the default; with
    waves of 2^16 points the tasks are cut into several pieces and the
    pieces spread over several waves), the phased pass as one chain of
    launches per task tile (option batch_grouped 0), and every point in one
    thread of the persistent kernel (option batch_phased 0).  The grouped
    modes keep the reference's retry loop (the default) or run a fixed budget
    (option batch_retry 0, which the other two modes need).  The 2->4 task
    with cuts rejects most points: its first iteration needs further rounds
    (the first draws ncalls points and a small margin), after which its draws
    are re-planned and a later iteration needs few if any."""
    # the 2->4 task spans two phased tiles (2^18 points each)
    tasks = [mc_task(2, 500.0, 20000, 20), mc_task(3, 1500.0, 5000, 30), mc_task(4, 1000.0, 265000, 25, cuts=True),
             mc_task(5, 800.0, 20000, 15)]
    retry = mode in ("grouped", "grouped_small_waves")
    ctx = ctx_factory()
    if mode.endswith("small_waves"):
        # waves on one stream: each reuses the buffers of the one before
        ctx.set_option("batch_wave_points", 1 << 16)
        ctx.set_option("batch_wave_streams", 1)
    ctx.set_option("batch_grouped", 0 if mode == "task_chains" else 1)
    ctx.set_option("batch_phased", 0 if mode == "one_kernel" else 1)
    ctx.set_option("batch_retry", 1 if retry else 0)
    _, infos = run_and_check(ctx, tasks, seed=11, iterations=2, retry=retry)
    assert (infos[0][0] > 2) == retry, infos
    l0 = ctx.launches
    _, info = ctx.batch_iterate(1, seed=11, adapt=True)
    launches = ctx.launches - l0
    if mode.startswith("grouped"):
        # a handful of launches per wave and round, not a chain per task tile
        assert info.retry_rounds <= 2, info.retry_rounds
        per_round = 30 if mode in ("grouped", "grouped_fixed") else 200
        assert launches < per_round * (1 + info.retry_rounds), launches


def test_retry_loop_needs_the_grouped_phased_pass(ctx_factory):
    from chili_b200.gpu import ChiliError
    ctx = ctx_factory()
    ctx.set_option("batch_retry", 1)
    ctx.set_option("batch_grouped", 0)
    with pytest.raises(ChiliError):
        ctx.batch_set([mc_task(2, 500.0, 1000, 20)])
    ctx.set_option("batch_retry", 0)
    ctx.batch_set([mc_task(2, 500.0, 1000, 20)])


def test_mixed_batch_matches_the_oracle(ctx_factory):
    """Camel and multichannel tasks in one launch, several iterations per
    call (one graph replay each): the same results as one call per
    iteration, and the oracle's."""
    rng = np.random.default_rng(8)
    tasks = [camel_task(rng, 3, 40000, 30), mc_task(2, 300.0, 10000, 20), camel_task(rng, 7, 777, 25),
             mc_task(5, 800.0, 4000, 15)]
    ctx = ctx_factory()
    ctx.set_option("batch_retry", 1)
    ctx.batch_set(tasks)
    st, info = ctx.batch_iterate(3, seed=21, adapt=True)
    want = [oracle_camel(t, 21 + k, 3) if t["kind"] == "camel" else oracle_mc(t, 21 + k, 3)
            for k, t in enumerate(tasks)]
    for k in range(len(tasks)):
        e, a = ctx.batch_get_grid(k)
        for it in range(3):
            st_o = want[k][it][0]
            assert st[it, k, 0] == st_o[0] and st[it, k, 5] == st_o[5], (k, it)
            assert rel(st[it, k, 3], st_o[3]) < (1e-11 if it == 0 else 1e-9), (k, it)
        check_task(k, st[2, k], e, a, want[k][2], 2)
    assert info.ms_per_iteration > 0


def test_batch_rejects_bad_tasks(ctx_factory):
    from chili_b200.gpu import ChiliError
    ctx = ctx_factory()
    rng = np.random.default_rng(1)
    bad = camel_task(rng, 3, 100, 20)
    bad["params"] = bad["params"][:-1]
    with pytest.raises(ChiliError):
        ctx.batch_set([bad])
    t = mc_task(2, 500.0, 100, 20)
    t["fkind"] = abi.CHILI_FUNC_CAMEL
    with pytest.raises(ChiliError):
        ctx.batch_set([t])
    with pytest.raises(ChiliError):
        ctx.batch_iterate(1)


def test_graph_recapture_on_changed_calls(ctx_factory):
    """Calls that change the iteration count (more stats slots) or switch
    adaptation off and on re-capture the iteration graph: the same results
    as one call per iteration on a second context."""
    rng = np.random.default_rng(12)
    tasks = [camel_task(rng, 4, 20000, 30), mc_task(3, 700.0, 8000, 20)]
    a, b = ctx_factory(), ctx_factory()
    a.batch_set(tasks)
    b.batch_set(tasks)
    plan = [(1, True), (2, False), (3, True), (1, False)]
    got, want = [], []
    for n, adapt in plan:
        st, _ = a.batch_iterate(n, seed=3, adapt=adapt)
        got += list(st)
        for _ in range(n):
            s1, _ = b.batch_iterate(1, seed=3, adapt=adapt)
            want.append(s1[0])
    assert len(got) == len(want) == 7
    for g, w in zip(got, want):
        assert np.array_equal(g[:, 0], w[:, 0]) and np.array_equal(g[:, 5], w[:, 5])
        assert np.max(rel(g[:, 3], w[:, 3])) < 1e-9
    for k in range(len(tasks)):
        ea, aa = a.batch_get_grid(k)
        eb, ab = b.batch_get_grid(k)
        assert np.max(rel(ea, eb)) < 1e-7 and np.max(rel(aa, ab)) < 1e-7
