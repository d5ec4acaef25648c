"""The C ABI without a GPU: the library loads and exports every function include/apo2.h
declares, the ctypes mirror agrees with the C layout of the option/stat structs, the C++
mirror of the reference interface (include/apo/gpu/algorithm.hpp) compiles and links, and
the host-only entry points behave. No call here reaches the device."""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "apo2.h")
COMPAT = os.path.join(ROOT, "include", "apo", "gpu", "algorithm.hpp")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^(?:const\s+)?\w+\s*\*?\s*(apo2_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    import apo_b200
    return apo_b200.load_library()


def test_header_declares_the_expected_surface():
    names = declared_functions()
    for must in ("apo2_create", "apo2_build", "apo2_get_vertices", "apo2_get_closed_edges", "apo2_get_topology",
                 "apo2_compute_diagram", "apo2_compute_full_diagram", "apo2_lbvh_build", "apo2_radix_sort_pairs",
                 "apo2_radix_sort_pairs_static", "apo2_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    import apo_b200
    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers exactly the header
    assert sorted(apo_b200.SIGNATURES) == names


def test_version_and_error_string(lib):
    assert lib.apo2_version().decode().startswith("apo2")
    assert isinstance(lib.apo2_last_error_string(), bytes)


def test_host_argument_checks_without_device(lib):
    import apo_b200
    # null handles and null outputs are rejected before any CUDA call
    assert lib.apo2_destroy(None) in (apo_b200.APO2_OK, 1)
    assert lib.apo2_get_stats(None, None) == 1
    assert lib.apo2_build(None, None, 1) == 1
    assert lib.apo2_create(None, 0, 1, 0, None, None) == 1
    assert lib.apo2_radix_sort_pairs_static(None, None, 0, None) == 1
    assert lib.apo2_certify(None, None, None, 0, 4, 0, None, None) == 1
    assert lib.apo2_topology_json(None, None, 0, None) == 1
    assert lib.apo2_batch_create(1, 4, None, None) == 1
    assert lib.apo2_batch_build(None, None, None, 0, None, None, None, None) == 1
    assert lib.apo2_batch_destroy(None) == 0
    # a shard index at or past the shard count is rejected before any CUDA call
    opt = apo_b200.Options()
    opt.struct_size = ctypes.sizeof(apo_b200.Options)
    opt.shard_index, opt.shard_count = 3, 3
    sites = (ctypes.c_float * 16)()
    handle = ctypes.c_void_p()
    assert lib.apo2_create(sites, 4, apo_b200.APO2_F32, apo_b200.APO2_HOST, ctypes.byref(opt), ctypes.byref(handle)) == 1
    assert b"shard" in lib.apo2_last_error_string()
    keys = ctypes.c_void_p(16)
    assert lib.apo2_radix_sort_pairs_static(keys, keys, (1 << 20) + 1, None) == 7  # APO2_ERR_TOO_LARGE
    assert lib.apo2_radix_sort_scratch_bytes(1 << 20) + 256 <= 256 + 12853760 + 4096


def _struct_layout_program() -> str:
    return r"""
#include <stddef.h>
#include <stdio.h>
#include "apo2.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
    printf("apo2_options %zu\n", sizeof(apo2_options));
    printf("apo2_stats %zu\n", sizeof(apo2_stats));
    F(apo2_options, k) F(apo2_options, edge_search) F(apo2_options, wait_limit) F(apo2_options, reserved)
    F(apo2_stats, vertex_records) F(apo2_stats, ms_bounds) F(apo2_stats, ms_output) F(apo2_stats, device_bytes)
    F(apo2_stats, uncertified)
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")
def test_ctypes_structs_match_c_layout(tmp_path):
    import apo_b200
    src = tmp_path / "layout.c"
    src.write_text(_struct_layout_program())
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                               text=True).stdout.split("\n") if line)
    assert int(out["apo2_options"]) == ctypes.sizeof(apo_b200.Options)
    assert int(out["apo2_stats"]) == ctypes.sizeof(apo_b200.Stats)
    for key, value in out.items():
        if "." in key:
            struct, member = key.split(".")
            cls = apo_b200.Options if struct == "apo2_options" else apo_b200.Stats
            assert getattr(cls, member).offset == int(value), key


COMPAT_PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "apo/gpu/algorithm.hpp"
#include "apo/gpu/cavity.hpp"

// instantiate the whole mirror so every member is type-checked against the C ABI
template class apo::gpu::AlgorithmGPU<16>;
template class apo::gpu::AlgorithmGPU<8>;

int main(int argc, char **) {
    std::printf("%s\n", apo2_version());
    std::vector<float> xyzr(4 * 2 * 32);
    if (apo2_generate_chains(2, 32, 0.05, 7, xyzr.data()) != APO2_OK) return 1;
    std::vector<apo::Real> sites(xyzr.begin(), xyzr.end());
    apo::ConstSpan<apo::Real> span{sites};
    if (span.size != sites.size()) return 2;
    // the cavity application's directions are computed on the host
    const std::vector<float> dirs = apo::gpu::getDirections(64);
    if (dirs.size() != 192 || dirs[0] != 0.f || dirs[1] != 0.f || dirs[2] != -1.f) return 3;
    if (argc > 5) {  // not taken here: the call sequence runs on a GPU in tests/test_gpu_compat_cpp.py
        apo::gpu::CavityDetection cavity{span};
        std::vector<float> loaded(xyzr.begin(), xyzr.end());
        auto ratios = cavity.getHitRatios(apo::ConstSpan<float>{loaded});
        auto found = cavity.filterVertices({cavity.vertexNb(), .5f, 5.f});
        std::printf("%zu %zu\n", ratios.size(), found.size());
        apo::gpu::AlgorithmGPU<16> algo{span};
        algo.build();
        auto full = algo.toHostFull(true);
        auto topo = algo.toTopology();
        auto diagram = apo::gpu::computeApolloniusDiagram(span);
        std::printf("%zu %zu %zu\n", full.vertices.size(), topo.bisectors.size(), diagram.verticesId.size());
    }
    std::printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ missing")
@pytest.mark.parametrize("real_size", [8, 4])
def test_compat_header_compiles_links_and_runs(lib, tmp_path, real_size):
    import apo_b200
    src = tmp_path / "compat.cpp"
    src.write_text(COMPAT_PROGRAM)
    exe = tmp_path / "compat"
    libdir = os.path.dirname(apo_b200.library_path())
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", f"-DAPO_REAL_SIZE={real_size}",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lapo2", f"-Wl,-rpath,{libdir}", "-Wl,--allow-shlib-undefined"], check=True)
    env = dict(os.environ)
    import nvidia.cuda_runtime as cr  # libcudart.so.12 for the loader
    env["LD_LIBRARY_PATH"] = os.path.join(list(cr.__path__)[0], "lib") + ":" + env.get("LD_LIBRARY_PATH", "")
    run = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    assert run.returncode == 0, run.stderr
    assert run.stdout.split()[-1] == "ok"


def test_generate_chains_is_deterministic_and_matches_the_python_generator(lib):
    from apo_b200 import generators
    a = np.empty((3 * 50, 4), np.float32)
    b = np.empty((3 * 50, 4), np.float32)
    assert lib.apo2_generate_chains(3, 50, 0.05, 11, a.ctypes.data) == 0
    assert lib.apo2_generate_chains(3, 50, 0.05, 11, b.ctypes.data) == 0
    assert np.array_equal(a, b)
    c = generators.protein_chains(3, atoms_per_chain=50, density=0.05, seed=11)
    assert np.array_equal(np.asarray(c, np.float32).reshape(-1, 4), a)
    # bonded neighbours sit 1.53 A apart, radii are van der Waals radii
    d = np.linalg.norm(np.diff(a[:50, :3], axis=0), axis=1)
    assert np.allclose(d, 1.53, atol=1e-3)
    assert a[:, 3].min() >= 1.0 and a[:, 3].max() <= 2.1
