"""The reference's results.chili checkpoints through the C ABI: a file written
by the reference (MultiChannel::SaveAs) loads into the GPU context with the
same grids and channel weights and is written back byte for byte; a file
written after GPU iterations loads into the reference (LoadFrom) with the GPU's
grids and best weights."""
import numpy as np
import pytest

from chili_b200 import abi, channels, workloads
from oracle import port, ref

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) absent")


def _ctx(ctx_factory, cs, bins):
    ctx = ctx_factory()
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, bins)
    ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    ctx.set_preprocess(abi.CHILI_PRE_FINITE)
    return ctx


@needs_ref
def test_reference_checkpoint_round_trip(ctx_factory, tmp_path):
    cs = channels.multichannel_2_to_4()
    params = workloads.mc_params(3000)
    R = ref.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    rng = np.random.default_rng(3)
    for _ in range(2):
        R.iterate(workloads.uniforms53(rng, (20000, R.ndims + 1)))
    p1 = tmp_path / "ref.chili"
    R.save(p1)
    ctx = _ctx(ctx_factory, cs, 50)
    p, results = ctx.load_checkpoint(p1)
    assert np.array_equal(ctx.get_grids(), R.get_grids())
    a_r, best_r, md_r = R.get_alpha()
    alpha, best, md = ctx.get_alpha()
    assert np.array_equal(best, best_r) and np.array_equal(alpha, best_r) and md == md_r
    assert p.ncalls == 3000 and p.nrefine == params.nrefine and p.beta == params.beta
    p2 = tmp_path / "gpu.chili"
    ctx.save_checkpoint(p2, p, results)
    assert p2.read_bytes() == p1.read_bytes()


@needs_ref
def test_gpu_checkpoint_loads_into_reference(ctx_factory, tmp_path):
    cs = channels.multichannel_2_to_4()
    params = workloads.mc_params(20_000)
    ctx = _ctx(ctx_factory, cs, 50)
    counter = 0
    for _ in range(2):
        st, info = ctx.multichannel_iterate(params, seed=5, counter=counter)
        counter += info.points_tried
    p3 = tmp_path / "gpu2.chili"
    ctx.save_checkpoint(p3, params, [st])
    R = ref.MultiChannel(cs, 50, params, abi.CHILI_FUNC_PROPAGATOR, channels.propagator_params())
    R.load(p3)
    assert np.array_equal(R.get_grids(), ctx.get_grids())
    a_r, best_r, md_r = R.get_alpha()
    alpha, best, md = ctx.get_alpha()
    assert np.array_equal(a_r, best) and np.array_equal(best_r, best) and md_r == md
    # a mismatching channel set is refused
    other = _ctx(ctx_factory, channels.multichannel_2_to_6(), 50)
    with pytest.raises(Exception):
        other.load_checkpoint(p3)
