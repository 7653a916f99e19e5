"""The GPU FSMapper as the reference's own plugin type.

chili::gpu::GpuFSMapper (include/chili_b200_mapper.hh) derives from the
reference's Mapper<FourVector> (Mapper.hh:37-39).  oracle/_ref/mapper_driver,
built against the unmodified reference headers and sources, puts it into
Channel<FourVector> objects of a reference Integrand and compares it with
the stock FSMapper (Channel.hh:15-33): per channel on random uniforms
(GeneratePoint momenta, GenerateWeight weights and the in/out uniform
buffer), then whole MultiChannel::operator() iterations of the reference
(MultiChannel.hh:196-251) over the two integrands from the same seed, then
a checkpoint written with the GPU mappers loaded back as stock FSMappers.
Bars as the other parity tests: p99 within 1e-12, NaN decisions identical,
the tails bounded by the conditioning of the inverse maps."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "mapper_driver")


def test_mapper_driver_is_built_with_the_reference():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build absent")
    assert os.access(DRIVER, os.X_OK)


@pytest.mark.gpu
def test_gpu_mapper_inside_the_reference_integrand(tmp_path):
    if not os.access(DRIVER, os.X_OK):
        pytest.skip("oracle/_ref/mapper_driver not built")
    out = subprocess.run([DRIVER, "300", "400", "2", str(tmp_path / "gpu_mappers.chili")], capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.splitlines()
    maps = [ln.split()[1:] for ln in lines if ln.startswith("MAP")]
    assert len(maps) == 9
    for ch, npts, gmax, gp99, wmax, wp99, rmax, nanmis in maps:
        assert int(nanmis) == 0, ch
        assert float(gp99) < 1e-12 and float(wp99) < 1e-12, (ch, gp99, wp99)
        assert float(gmax) < 1e-9 and float(wmax) < 1e-6 and float(rmax) < 1e-6, (ch, gmax, wmax, rmax)
    iters = [ln.split()[1:] for ln in lines if ln.startswith("ITER")]
    assert len(iters) == 2
    for k, n, ms, mg, vs, vg in iters:
        assert int(float(n)) >= 400
        assert abs(float(mg) - float(ms)) <= 1e-10 * abs(float(ms)), (k, ms, mg)
        assert abs(float(vg) - float(vs)) <= 1e-8 * abs(float(vs)), (k, vs, vg)
    assert "SAVE ok" in lines
