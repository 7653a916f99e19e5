"""Pins the C restatement (oracle/port) to the reference.

1. Against the committed fixtures made from the compiled reference
   (tests/golden/make_golden.py): always runs, bit-exact.
2. Against the live reference build (oracle/_ref) on fresh seeded inputs when
   that build is present: bit-exact.
"""
import os

import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from oracle import port, ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.fixture(scope="module")
def g():
    return dict(np.load(os.path.join(GOLDEN, "grids.npz")))


@pytest.fixture(scope="module")
def m():
    return dict(np.load(os.path.join(GOLDEN, "multichannel_2to4.npz")))


def test_port_grid_primitives_match_golden(g):
    e = g["grid_edges"]
    x, jac = port.am_map(e, g["grid_u"])
    assert eq(x, g["grid_x"]) and eq(jac, g["grid_jac"])
    w, b = port.am_weight(e, g["grid_xw"])
    assert eq(b, g["grid_bin"])
    ok = ~np.isnan(g["grid_w"])  # the reference driver reports NaN where it would read outside its table
    assert eq(w[ok], g["grid_w"][ok])
    assert eq(port.am_adapt(e, 1.5, g["grid_train"]), g["grid_adapted"])
    for k in (2, 3, 4):
        assert eq(port.am_split(e, k), g[f"grid_split{k}"])


def test_port_vegas_iteration_matches_golden(g):
    st, tr, e2 = port.vegas_iterate(g["grid_edges"], 1.5, g["vegas_params"], g["vegas_u"])
    assert eq(st.as_tuple(), g["vegas_stats"])
    assert eq(tr, g["vegas_train"])
    assert eq(e2, g["vegas_edges_after"])


def test_port_channel_selection_matches_golden(g):
    assert eq(port.select(g["select_alpha"], g["select_v"]), g["select_ich"])


@pytest.fixture(scope="module")
def mc2():
    return channels.multichannel_2_to_4()


def test_port_fsmapper_matches_golden(m, mc2):
    O = port.MultiChannel(mc2, 100, workloads.mc_params(400), abi.CHILI_FUNC_PROPAGATOR,
                          channels.propagator_params())
    for ch in range(mc2.nch):
        mom = O.fsm_generate(ch, m["fsm_x"][ch])
        assert eq(mom, m["fsm_mom"][ch]), ch
        w, xi = O.fsm_weight(ch, m["fsm_mom"][ch])
        assert eq(w, m["fsm_w"][ch]) and eq(xi, m["fsm_xinv"][ch]), ch


def test_port_multichannel_iterations_match_golden(m, mc2):
    O = port.MultiChannel(mc2, 100, workloads.mc_params(400), abi.CHILI_FUNC_PROPAGATOR,
                          channels.propagator_params())
    O.set_grids(m["mc_edges0"])
    for it in range(3):
        st, info = O.iterate(m["mc_u"][it], guard=True)
        assert eq(st.as_tuple(), m["mc_stats"][it]), it
        assert eq([info.points_tried, info.rejected_pre, info.rejected_nan, info.weight_max,
                   info.nonfinite_alpha_terms], m["mc_info"][it]), it
        a, b, md = O.get_alpha()
        assert eq(a, m["mc_alpha"][it]) and eq(b, m["mc_best"][it]) and eq([md], m["mc_min_diff"][it])
        h, atr = O.training()
        assert eq(atr, m["mc_atrain"][it])
    assert eq(O.get_grids(), m["mc_grids"])
    assert eq(h, m["mc_hist"])


def test_port_combined_weight_and_evaluate_match_golden(m, mc2):
    O = port.MultiChannel(mc2, 100, workloads.mc_params(400), abi.CHILI_FUNC_PROPAGATOR,
                          channels.propagator_params())
    O.set_grids(m["cw_grids"])
    O.set_alpha(m["cw_alpha"])
    w, dens, xi = O.weight(m["cw_mom"], m["cw_ich"])
    assert eq(w, m["cw_w"]) and eq(dens, m["cw_dens"]) and eq(xi, m["cw_x"])
    for k, ch in enumerate((0, 7, 12)):
        assert eq(O.evaluate_batch(ch, m["eval_u"]), m["eval_out"][k])


needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) absent")


@needs_ref
def test_port_matches_live_reference_on_fresh_inputs():
    rng = np.random.default_rng(99)
    cs = channels.multichannel_2_to_6()
    params = workloads.mc_params(300)
    R = ref.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR_TOP2, channels.propagator_params())
    O = port.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR_TOP2, channels.propagator_params())
    nd = R.ndims
    assert nd == 16
    for ch in range(0, cs.nch, 4):
        x = workloads.uniforms53(rng, (300, nd))
        m1, m2 = R.fsm_generate(ch, x), O.fsm_generate(ch, x)
        assert eq(m1, m2), ch
        assert eq(R.fsm_weight(ch, m1)[0], O.fsm_weight(ch, m1)[0]), ch
    for it in range(2):
        u = workloads.uniforms53(rng, (3000, nd + 1))
        s1, i1 = R.iterate(u)
        s2, i2 = O.iterate(u)
        assert eq(s1.as_tuple(), s2.as_tuple()) and i1.points_tried == i2.points_tried
        assert eq(R.get_alpha()[0], O.get_alpha()[0])
        assert eq(R.get_grids(), O.get_grids())


@needs_ref
def test_cut_preprocess_port_matches_reference_driver():
    """CHILI_PRE_CUTS: the port and the reference driven with the same
    PreProcess reject the same points and agree bit for bit."""
    rng = np.random.default_rng(7)
    cs = channels.multichannel_2_to_4()
    params = workloads.mc_params(2000)
    R = ref.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    O = port.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    R.set_cuts(1000.0)
    O.set_cuts(1000.0)
    for it in range(2):
        u = workloads.uniforms53(rng, (40000, R.ndims + 1))
        s1, i1 = R.iterate(u)
        s2, i2 = O.iterate(u)
        assert i1.points_tried == i2.points_tried and i1.rejected_pre == i2.rejected_pre
        if it == 0:  # uniform grids: the cuts remove most points (adapted grids avoid them)
            assert i1.rejected_pre > i1.points_tried // 2
        assert eq(s1.as_tuple(), s2.as_tuple())
        assert eq(R.get_alpha()[0], O.get_alpha()[0])


@needs_ref
def test_unguarded_alpha_goes_nan_like_the_reference():
    """Without the guard both oracles propagate the non-finite alpha-training
    terms (MultiChannel.hh:176) and end the first iteration with NaN alpha."""
    rng = np.random.default_rng(5)
    cs = channels.multichannel_2_to_4()
    params = workloads.mc_params(2000)
    R = ref.MultiChannel(cs, 100, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    O = port.MultiChannel(cs, 100, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    u = workloads.uniforms53(rng, (6000, R.ndims + 1))
    s1, _ = R.iterate(u, guard=False)
    s2, _ = O.iterate(u, guard=False)
    assert eq(s1.as_tuple(), s2.as_tuple())
    a1, a2 = R.get_alpha()[0], O.get_alpha()[0]
    assert eq(a1, a2)
    assert np.isnan(a1).all()


def test_port_philox_is_the_published_algorithm():
    """Philox4x32-10 restated in Python from Salmon et al. (SC'11) agrees with
    the C port's uniforms."""
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    mask = 0xFFFFFFFF

    def philox(c, k):
        c = list(c)
        k0, k1 = k
        for _ in range(10):
            p0, p1 = M0 * c[0], M1 * c[2]
            c = [((p1 >> 32) ^ c[1] ^ k0) & mask, p1 & mask, ((p0 >> 32) ^ c[3] ^ k1) & mask, p0 & mask]
            k0, k1 = (k0 + W0) & mask, (k1 + W1) & mask
        return c

    seed, ctr0, n, d = 0x123456789ABCDEF, 2 ** 32 - 3, 7, 11
    got = port.philox_uniforms(seed, ctr0, n, d)
    for i in range(n):
        k = ctr0 + i
        for q in range((d + 1) // 2):
            r = philox([q, k & mask, k >> 32, 0], [seed & mask, seed >> 32])
            u0 = ((r[0] << 21) | (r[1] >> 11)) * 2.0 ** -53
            u1 = ((r[2] << 21) | (r[3] >> 11)) * 2.0 ** -53
            assert got[i, 2 * q] == u0
            if 2 * q + 1 < d:
                assert got[i, 2 * q + 1] == u1
    assert (got >= 0).all() and (got < 1).all()


def test_point_values_and_accept_stream():
    """The oracle's per-point values (input of the unweighting stage) are the
    fixed-budget iteration's values: same sum and nonzero count; stream 0 of
    the stream generator is the points' generator."""
    cs = workloads.channel_set(4)
    params = workloads.mc_params(3000)
    O = port.MultiChannel(cs, 20, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    O.set_cuts(cs.sqrts)
    u = port.philox_uniforms(9, 100, 3000, O.ndims + 1)
    assert np.array_equal(u, port.philox_stream_uniforms(9, 100, 3000, O.ndims + 1, 0))
    assert not np.array_equal(u[:, :2], port.philox_stream_uniforms(9, 100, 3000, 2, 1))
    val, ich, mom = O.point_values(u)
    O.set_fixed_budget(True)
    st, info = O.iterate(u)
    assert st.n == 3000 and st.n_finite == np.count_nonzero(val)
    assert abs(st.sum - val.sum()) <= 1e-13 * abs(val).sum()
