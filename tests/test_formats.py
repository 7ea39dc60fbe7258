"""gen_N.txt / shared_data.txt readers and writers (reference formats)."""
import numpy as np

from symbolic_regression_gpu_b200 import formats, synth


def test_gen_file_round_trip(tmp_path):
    w = synth.plain_workload(seed=5, E=40, N=64)
    path = tmp_path / "gen_0.txt"
    formats.write_gen_file(str(path), w.population, w.num_vars, w.num_dps, "shared_data.txt")
    pop, nv, nd, files = formats.read_gen_file(str(path))
    assert (pop.tokens == w.population.tokens).all()
    assert (pop.values == w.population.values).all()
    assert (pop.offsets == w.population.offsets).all()
    assert set(nv) == {w.num_vars} and set(nd) == {w.num_dps}
    assert set(files) == {"shared_data.txt"}


def test_reference_layout_is_parsed(tmp_path):
    # Two expressions in the reference layout (one header line, then per
    # expression: counts / tokens / values / data file).
    text = ("2\n1\n1000\n5\n1 0 4 0 -1\n0 3.0 0 1.0 0\ndata/a\n"
            "3\n1000\n7\n4 3 -1 -1 4 -1 0\n0 0 0 1 0 2 1.0\ndata/b\n")
    p = tmp_path / "g.txt"
    p.write_text(text)
    pop, nv, nd, files = formats.read_gen_file(str(p))
    assert pop.num_exprs == 2 and nv == [1, 3] and nd == [1000, 1000]
    assert list(pop.expr(0)[0]) == [1, 0, 4, 0, -1]
    assert list(pop.expr(1)[1]) == [0, 0, 0, 1, 0, 2, 1.0]
    assert files == ["data/a", "data/b"]


def test_shared_data_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    X = rng.uniform(-5, 5, size=(4, 100)).astype(np.float32)
    p = tmp_path / "shared_data.txt"
    formats.write_shared_data(str(p), X)
    Y = formats.read_shared_data(str(p), 3)
    assert Y.shape == X.shape
    assert (Y.astype(np.float32) == X).all()
    Z = formats.read_shared_data(str(p), 3, num_dps=10)
    assert Z.shape == (4, 10)
