"""The C-ABI library (no GPU needed): it loads, exports every entry point that
include/chili_gpu.h declares, its structs have the header's layout, it fails
cleanly without a device, and its host-side channel validation works."""
import ctypes as C
import os
import re
import subprocess

import pytest

from chili_b200 import abi, channels, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chili_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|uint64_t|const char \*)\s*(chili_gpu_\w+)\s*\(", src, re.M)))


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_symbol():
    lib = gpu.load()
    names = declared_functions()
    assert len(names) >= 25
    syms = exported_symbols(gpu.LIB_PATH)
    missing = [n for n in names if n not in syms]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)
    # and the binding declares a signature for each of them
    assert set(names) <= set(gpu.EXPORTED)


def test_struct_layouts_match_the_header(tmp_path):
    """Compiles a probe against the header and compares sizes and offsets with
    the ctypes mirror."""
    probe = tmp_path / "layout.c"
    probe.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "chili_gpu.h"
#define S(t) printf(#t " %zu\n", sizeof(t));
#define O(t, f) printf(#t "." #f " %zu\n", offsetof(t, f));
int main(void) {
  S(chili_particle_info) S(chili_decay) S(chili_channel_desc) S(chili_idx_value)
  S(chili_pid_pair_value) S(chili_cuts) S(chili_stats) S(chili_multichannel_params) S(chili_mc_iter_info)
  S(chili_flow_params) S(chili_flow_iter_info) O(chili_flow_params, init_seed) O(chili_flow_params, depth) O(chili_flow_iter_info, unweighting_efficiency)
  O(chili_multichannel_params, should_optimize) O(chili_multichannel_params, grid_alpha)
  O(chili_cuts, etamax) O(chili_mc_iter_info, weight_max) O(chili_mc_iter_info, points_weighted) O(chili_mc_iter_info, chunks)
  S(chili_task) S(chili_batch_info) O(chili_task, ncalls) O(chili_task, params) O(chili_task, descs)
  O(chili_task, sqrts) O(chili_task, n_ext) O(chili_task, pre_cuts) O(chili_batch_info, points) O(chili_batch_info, retry_rounds)
  return 0;
}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(probe), "-o", str(exe)], check=True)
    got = dict(ln.rsplit(" ", 1) for ln in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    mirror = {"chili_particle_info": abi.ParticleInfo, "chili_decay": abi.Decay, "chili_channel_desc": abi.ChannelDesc,
              "chili_idx_value": abi.IdxValue, "chili_pid_pair_value": abi.PidPairValue, "chili_cuts": abi.Cuts,
              "chili_stats": abi.Stats, "chili_multichannel_params": abi.MultiChannelParams,
              "chili_mc_iter_info": abi.MCIterInfo, "chili_flow_params": abi.FlowParams,
              "chili_flow_iter_info": abi.FlowIterInfo, "chili_task": abi.Task, "chili_batch_info": abi.BatchInfo}
    for name, cls in mirror.items():
        assert int(got[name]) == C.sizeof(cls), name
    assert int(got["chili_multichannel_params.should_optimize"]) == abi.MultiChannelParams.should_optimize.offset
    assert int(got["chili_multichannel_params.grid_alpha"]) == abi.MultiChannelParams.grid_alpha.offset
    assert int(got["chili_cuts.etamax"]) == abi.Cuts.etamax.offset
    assert int(got["chili_mc_iter_info.weight_max"]) == abi.MCIterInfo.weight_max.offset
    assert int(got["chili_mc_iter_info.points_weighted"]) == abi.MCIterInfo.points_weighted.offset
    assert int(got["chili_mc_iter_info.chunks"]) == abi.MCIterInfo.chunks.offset
    assert int(got["chili_flow_params.init_seed"]) == abi.FlowParams.init_seed.offset
    assert int(got["chili_flow_params.depth"]) == abi.FlowParams.depth.offset
    assert int(got["chili_flow_iter_info.unweighting_efficiency"]) == abi.FlowIterInfo.unweighting_efficiency.offset
    for f in ("ncalls", "params", "descs", "sqrts", "n_ext", "pre_cuts"):
        assert int(got["chili_task." + f]) == getattr(abi.Task, f).offset, f
    assert int(got["chili_batch_info.points"]) == abi.BatchInfo.points.offset
    assert int(got["chili_batch_info.retry_rounds"]) == abi.BatchInfo.retry_rounds.offset


def test_header_limits_match_the_mirror():
    src = open(HEADER).read()
    for name in ("CHILI_MAX_EXT", "CHILI_MAX_DIMS", "CHILI_MAX_CHANNELS", "CHILI_MAX_BINS",
                 "CHILI_MAX_INTEGRAND_PARAMS"):
        v = int(re.search(rf"#define {name} (\d+)", src).group(1))
        assert v == getattr(abi, name), name


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda(), reason="checks the no-device error path")
def test_create_without_a_device_fails_cleanly():
    lib = gpu.load()
    h = C.c_void_p()
    rc = lib.chili_gpu_create(0, C.byref(h))
    assert rc == abi.CHILI_ERR_CUDA
    assert not h.value
    assert b"device" in lib.chili_gpu_last_error(None).lower()
    with pytest.raises(gpu.ChiliError):
        gpu.Context(0)


def test_null_arguments_are_rejected_without_a_context():
    lib = gpu.load()
    assert lib.chili_gpu_create(0, None) == abi.CHILI_ERR_INVALID_ARG
    assert lib.chili_gpu_destroy(None) == abi.CHILI_OK
    assert lib.chili_gpu_set_grids(None, None, 1, 1, 2) == abi.CHILI_ERR_INVALID_ARG
    assert lib.chili_gpu_launch_count(None) == 0


@pytest.mark.parametrize("build", [channels.multichannel_2_to_4, channels.multichannel_2_to_6,
                                   lambda: channels.multichannel_2_to_n(3, 500.0),
                                   lambda: channels.multichannel_2_to_n(5, 2000.0)])
def test_workload_channel_sets_validate(build):
    cs = build()
    assert gpu.check_channels(cs) == ""


def _mutated(mutate):
    cs = channels.multichannel_2_to_4()
    chans = [(list(i), list(d)) for i, d in cs.channels]
    cuts = {"sexternal": [0.0] * 4, "deltaR": {}, "smin": {}, "ptmin": {}, "etamax": {}}
    cuts = channels.default_cuts(channels.process_2_to_n(4))
    for info, decs in chans:
        for d in decs:
            cuts["ptmin"].setdefault(d.parent.idx, 0.0)
            cuts["etamax"].setdefault(d.parent.idx, 99.0)
    mutate(chans, cuts)
    return abi.ChannelSet(chans, cuts, 1000.0, 6)


def test_invalid_channel_descriptions_are_rejected():
    # a t-channel list that misses an outgoing leg
    cs = _mutated(lambda ch, cu: ch[6][0].pop(0))
    assert "cover" in gpu.check_channels(cs) or "uniform" in gpu.check_channels(cs)
    # a decaying current without its decay
    cs = _mutated(lambda ch, cu: ch[0][1].clear())
    assert gpu.check_channels(cs) != ""
    # a missing ptmin entry (the reference's .at() would throw)
    def drop_pt(ch, cu):
        del cu["ptmin"][4]
    assert "ptmin" in gpu.check_channels(_mutated(drop_pt))
    # overlapping t-channel entries
    def dup(ch, cu):
        ch[6][0].append(ch[6][0][0])
    assert gpu.check_channels(_mutated(dup)) != ""
