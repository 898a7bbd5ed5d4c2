"""The C++ host interface (include/qsketch_b200.hpp) compiles against the C ABI and, on a
GPU, gives the oracle's estimates."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import qsketch_b200 as qs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "host_api_driver.cpp")


def build(tmp_path):
    exe = str(tmp_path / "host_api_driver")
    lib_dir = os.path.dirname(qs.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", SRC, "-o", exe, "-I", os.path.join(ROOT, "include"),
           "-I", "/usr/local/cuda/include", "-L", lib_dir, "-lqsketch", "-L", "/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{lib_dir}", "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_cpp_header_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_cpp_driver_matches_oracle(tmp_path, gpu):
    exe = build(tmp_path)
    rng = np.random.default_rng(9)
    keys = (rng.zipf(1.2, 1 << 20) % 40000).astype(np.uint32) * np.uint32(2654435761)
    queries = np.unique(keys)[:20000]
    masks = qs.generate_hashmask(1021, 32, 3, 4, 4)
    kf, qf, mf, of = (str(tmp_path / n) for n in ("k.bin", "q.bin", "m.bin", "o.bin"))
    keys.tofile(kf)
    queries.tofile(qf)
    masks.tofile(mf)
    seed = 2654435769
    r = subprocess.run([exe, kf, qf, mf, of, "4093", "4096", str(seed)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + r.stdout
    got = np.fromfile(of, np.uint32)
    orc = oracle.Msws(4093, 4096, seed, masks)
    orc.insert(keys)
    assert np.array_equal(got, orc.query(queries))
