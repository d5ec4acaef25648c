"""The C++ mirror of the reference's interface (include/apo/gpu/algorithm.hpp, cavity.hpp) run on
a GPU: a program written in the reference's call sequence -- AlgorithmGPU<16>{sites}.build(),
toHostFull(true), toTopology(), computeApolloniusDiagram(sites), and the cavity application's
calls -- is compiled against the headers, linked with libapo2.so and run on the reference's
precision cloud prec1; its output must equal the reference's own dump of that cloud."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests import helpers as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "apo/gpu/algorithm.hpp"
#include "apo/gpu/cavity.hpp"

int main(int argc, char ** argv) {
    if (argc < 3) return 1;
    std::FILE * f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<float> raw;
    float v;
    while (std::fread(&v, sizeof(float), 1, f) == 1) raw.push_back(v);
    std::fclose(f);
    std::vector<apo::Real> sites(raw.begin(), raw.end());
    apo::ConstSpan<apo::Real> span{sites};

    apo::gpu::AlgorithmGPU<16> algo{span};
    algo.build();
    const auto full = algo.toHostFull(true);
    const auto topo = algo.toTopology();
    const auto diagram = apo::gpu::computeApolloniusDiagram(span);

    apo::gpu::CavityDetection cavity{span};
    const auto ratios = cavity.getHitRatios(apo::ConstSpan<float>{raw});
    const auto found = cavity.filterVertices({cavity.vertexNb(), .5f, 5.f});

    std::FILE * o = std::fopen(argv[2], "wb");
    const uint64_t counts[5] = {full.verticesId.size(), topo.quadrisectors.size(), topo.trisectors.size(),
                                topo.bisectors.size(), diagram.verticesId.size()};
    std::fwrite(counts, sizeof(counts), 1, o);
    std::fwrite(full.verticesId.data(), sizeof(uint32_t), full.verticesId.size(), o);
    std::fwrite(full.vertices.data(), sizeof(apo::Real), full.vertices.size(), o);
    std::fwrite(topo.quadrisectors.data(), sizeof(uint32_t), topo.quadrisectors.size(), o);
    std::fwrite(topo.trisectors.data(), sizeof(uint32_t), topo.trisectors.size(), o);
    std::fwrite(topo.bisectors.data(), sizeof(uint32_t), topo.bisectors.size(), o);
    std::fwrite(diagram.verticesId.data(), sizeof(uint32_t), diagram.verticesId.size(), o);
    std::fclose(o);
    std::printf("%zu %zu\n", ratios.size(), found.size());
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ missing")
def test_cpp_mirror_runs_the_reference_call_sequence(tmp_path):
    import apo_b200
    sites = H.sites_for("prec1").astype(np.float32)
    golden = H.load_golden("prec1")
    src = tmp_path / "run.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "run"
    libdir = os.path.dirname(apo_b200.library_path())
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lapo2", f"-Wl,-rpath,{libdir}", "-Wl,--allow-shlib-undefined"], check=True)
    inp = tmp_path / "sites.f32"
    sites.tofile(inp)
    out = tmp_path / "out.bin"
    env = dict(os.environ)
    import nvidia.cuda_runtime as cr  # libcudart.so.12 for the loader
    env["LD_LIBRARY_PATH"] = os.path.join(list(cr.__path__)[0], "lib") + ":" + env.get("LD_LIBRARY_PATH", "")
    run = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, env=env, timeout=300)
    assert run.returncode == 0, run.stderr
    raw = out.read_bytes()
    counts = np.frombuffer(raw[:40], dtype=np.uint64)
    at = 40

    def take(dtype, count):
        nonlocal at
        a = np.frombuffer(raw[at:at + np.dtype(dtype).itemsize * int(count)], dtype=dtype)
        at += a.nbytes
        return a

    ids = take(np.uint32, counts[0])
    pos = take(np.float64, counts[0])
    quad = take(np.uint32, counts[1])
    tri = take(np.uint32, counts[2])
    bi = take(np.uint32, counts[3])
    free_ids = take(np.uint32, counts[4])
    assert np.array_equal(ids, golden["vertices_id"])
    assert H.rel_err(pos, golden["vertices_pos"]) <= 1e-9
    assert np.array_equal(quad, golden["topo_quad"])
    assert np.array_equal(tri, golden["topo_tri"])
    assert np.array_equal(bi, golden["topo_bi"])
    assert np.array_equal(free_ids, golden["vertices_id"])
    n_ratios, n_found = map(int, run.stdout.split())
    assert n_ratios == counts[0] // 4 and 0 <= n_found <= n_ratios
