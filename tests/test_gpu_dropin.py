"""The reference evolution loop (src/cleaned/cl_sr_system.cpp, compiled
unchanged into oracle/_ref/) linked against libsr_eval.so."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from symbolic_regression_gpu_b200 import formats, synth

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def _best_mses(stdout):
    return [float(m) for m in re.findall(r"Best MSE: ([-+0-9.eEinfa]+)", stdout)]


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_BIN, "cl_sr_opt")),
                    reason="reference loop not built (make -C oracle ref)")
@pytest.mark.parametrize("variant", ["cl_sr_opt", "cl_sr_simple"])
def test_reference_loop_runs_on_this_library(tmp_path, variant):
    w = synth.plain_workload(seed=41, E=8, N=4000)
    formats.write_shared_data(str(tmp_path / "shared_data.txt"), w.X)
    formats.write_gen_file(str(tmp_path / "gen_0.txt"), w.population, w.num_vars, w.num_dps,
                           str(tmp_path / "shared_data.txt"))
    args = ["300", "4", str(tmp_path), "4000", "7"]
    env = dict(os.environ, THREADS="4")
    gpu = subprocess.run([os.path.join(REF_BIN, variant)] + args, capture_output=True, text=True,
                         timeout=300, cwd=str(tmp_path), env=env)
    assert gpu.returncode == 0, gpu.stderr[-2000:]
    cpu = subprocess.run([os.path.join(REF_BIN, "cl_sr_cpu")] + args, capture_output=True,
                         text=True, timeout=300, cwd=str(tmp_path), env=env)
    assert cpu.returncode == 0, cpu.stderr[-2000:]
    g, c = _best_mses(gpu.stdout), _best_mses(cpu.stdout)
    assert len(g) == 4 and len(c) == 4
    best = re.findall(r"Best Expr: (.*)", gpu.stdout)[:1] + re.findall(r"Best Expr: (.*)",
                                                                      cpu.stdout)[:1]
    print(f"{variant} gen-0 best MSE {g[0]} vs CPU {c[0]}; {best}")
    # Generation 0 is the same seeded population on both evaluators.  The loop
    # prints 6 significant digits, and a well-fitting expression amplifies the
    # ulp differences of CUDA's vs glibc's transcendentals: 1e-4 relative.
    assert abs(g[0] - c[0]) <= 1e-4 * max(abs(c[0]), 1e-6), (g[0], c[0], best)
