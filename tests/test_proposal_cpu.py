"""CPU checks of the k-proposal oracle (oracle/mlp_oracle.py), the checker of the GPU training
kernels: its gradient formulas against central differences, its bf16 rounding against torch's,
and the model struct layout against the C header."""
import ctypes

import numpy as np


def test_oracle_gradient_formulas_match_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(0)
    x = rng.normal(0, 1, (64, 16))
    y = rng.uniform(0, 4, 64)
    params = rng.normal(0, 0.3, M.N_PARAMS)
    g = M.analytic_float64(params, x, y)
    for idx in rng.choice(M.N_PARAMS, 60, replace=False).tolist() + [M.N_PARAMS - 1]:
        fd = M.finite_difference(params, x, y, idx, h=1e-5)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(g[idx]), (idx, fd, g[idx])


def test_bf16_rounding_matches_torch():
    import torch

    from oracle import mlp_oracle as M
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-3, 1000), [0.0, -0.0, 1.0, 3.0e38]]).astype(np.float32)
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(M.bf16_round(a), ref)


def test_proposal_struct_matches_the_header(tmp_path):
    import os
    import shutil
    import subprocess

    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("gcc missing")
    from apo_b200 import proposal as P
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "p.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "apo2.h"\nint main(void){printf("%zu %zu %zu %zu\\n",'
                   ' sizeof(apo2_proposal), offsetof(apo2_proposal, margin), offsetof(apo2_proposal, w1),'
                   ' offsetof(apo2_proposal, w3)); return 0;}\n')
    exe = tmp_path / "p"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    size, margin, w1, w3 = map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split())
    assert size == ctypes.sizeof(P.Proposal)
    assert margin == P.Proposal.margin.offset and w1 == P.Proposal.w1.offset and w3 == P.Proposal.w3.offset
    assert P.PARAMS == 5313
