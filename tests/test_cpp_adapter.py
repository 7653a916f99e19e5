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


def _build_vegas_driver(tmp_path):
    exe = tmp_path / "vegas_optimize"
    lib_dir = os.path.join(ROOT, "chili_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "vegas_optimize.cc"), "-L", lib_dir, "-lchili_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    return exe


def test_vegas_optimize_driver_compiles(tmp_path):
    assert _build_vegas_driver(tmp_path).exists()


@pytest.mark.gpu
def test_vegas_optimize_with_refine_matches_the_reference(tmp_path):
    """chili::gpu::Vegas::Optimize (C++ adapter, GPU) against the reference's
    own Vegas::Optimize (Vegas.cc:54-69) on the reference's own uniform
    stream (Random seeded with 42): the 4-d camel from 10 bins and 2000
    calls, Refine every 2 iterations (Vegas.cc:64-67: grid split in two,
    ncalls doubled), until the pooled error is below 0.5% after at least 5
    iterations.  Iteration count, calls per iteration, final bins and ncalls
    are equal; each iteration's sum and the pooled result agree to 1e-10
    relative and the final grid to 1e-10 (CUDA's exp and glibc's differ in
    the last ulp for some points, and the grids adapt on the sums)."""
    import numpy as np
    from chili_b200 import workloads
    from oracle import binding as B
    dims, bins, ncalls, nrefine, tol, nitn, alpha, seed = 4, 10, 2000, 2, 5e-3, 5, 1.5, 42
    camel = np.asarray(workloads.camel_params(dims), dtype=np.float64)
    r = B.vegas_optimize(dims, bins, alpha, camel, seed, ncalls, nrefine, tol, tol, nitn)
    assert r["n_iterations"] >= 5 and r["bins"] >= 4 * bins  # Refine fired at least twice
    total = int(sum(it[0] for it in r["iterations"])) * dims
    u = B.random_uniforms(seed, total)
    (tmp_path / "u.bin").write_bytes(u.tobytes())
    (tmp_path / "p.bin").write_bytes(camel.tobytes())
    exe = _build_vegas_driver(tmp_path)
    out = subprocess.run([str(exe), str(tmp_path / "u.bin"), str(tmp_path / "p.bin"), str(tmp_path / "e.bin"),
                          str(dims), str(bins), str(ncalls), str(nrefine), str(tol), str(tol), str(nitn),
                          str(alpha)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    iters = [ln.split()[1:] for ln in lines if ln.startswith("ITER")]
    res = [ln.split()[1:] for ln in lines if ln.startswith("RESULT")][-1]
    assert int(res[0]) == r["n_iterations"] == len(iters)
    assert int(res[1]) == r["bins"] and int(res[2]) == r["ncalls"]
    assert int(res[5]) == total  # every uniform consumed, in order
    for (n, s, s2), ref_it in zip(iters, r["iterations"]):
        assert int(n) == int(ref_it[0])
        assert abs(float(s) - ref_it[3]) <= 1e-10 * abs(ref_it[3])
        assert abs(float(s2) - ref_it[4]) <= 1e-10 * abs(ref_it[4])
    pooled = r["pooled"]
    mean_r = pooled[3] / pooled[0]
    assert abs(float(res[3]) - mean_r) <= 1e-10 * abs(mean_r)
    edges = np.frombuffer((tmp_path / "e.bin").read_bytes(), dtype=np.float64).reshape(dims, r["bins"] + 1)
    assert np.max(np.abs(edges - r["edges"])) < 1e-10


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
