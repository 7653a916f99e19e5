"""The C++ adapters (include/chili_b200.hh): a reference-style driver
(examples/multichannel_2to4.cc) compiles against them here and runs on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = tmp_path / "mc2to4"
    lib_dir = os.path.join(ROOT, "chili_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "examples", "multichannel_2to4.cc"), "-L", lib_dir, "-lchili_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    return exe


def test_cpp_driver_compiles_and_links(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_driver_runs(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([str(exe), "4"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("RESULT")][-1]
    _, mean, err, calls = line.split()
    mean, err = float(mean), float(err)
    assert mean > 0 and err > 0 and err / mean < 0.05
    assert int(calls) >= 4 * 200000


def test_cpp_construct_channels_runs_on_the_host(tmp_path):
    """chili::gpu::ConstructChannels with a std::function model (host code,
    no GPU): the same channels as the Python binding of the same call."""
    exe = tmp_path / "construct"
    lib_dir = os.path.join(ROOT, "chili_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "examples", "construct_channels.cc"), "-L", lib_dir, "-lchili_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), "2"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    n = int(lines[0].split()[1])
    assert lines[1] == "CHECK ok"

    from chili_b200 import gpu

    def comb(a, b):
        if a == -b and a != 0 and abs(a) not in (22, 23):
            return [22, 23]
        if b in (22, 23):
            return [a]
        if a in (22, 23):
            return [b]
        return []
    cs = gpu.construct_channels([11, -11, 13, -13, 22], comb, {11: 0, 13: 0, 22: 0, 23: 91.1876},
                                {11: 0, 13: 0, 22: 0, 23: 2.4952}, 1000.0, smax=2)
    assert n == cs.nch > 0
