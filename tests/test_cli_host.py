"""The reference-compatible command line and TSV report, on the CPU.

cli.main dispatches like cuda/main.cpp:9-147: 13 / 15 arguments (program name included) sweep
every block shape in 2D / 3D, 15 / 18 run one block shape, anything else prints the usage.  The
benchmark object is replaced by a recorder here, so no GPU is needed.  results_tsv follows
cuda/benchmark.cpp:354-428: per block shape the mean over launches of Flop/s and Lup/s, their
population standard deviations, the launch count and the total time.
"""

import math

import pytest

from threadcoarsenedstencilgenerator_b200 import benchmark as B
from threadcoarsenedstencilgenerator_b200 import cli


class Recorder:
    made = []

    def __init__(self, neighbourhood, dim, align, cl, coeff, orient, rng, coarsening, grid, max_time,
                 precision="f64"):
        self.args = dict(neighbourhood=neighbourhood, dim=dim, align=align, cl=cl, coeff=coeff, orient=orient,
                         rng=rng, coarsening=coarsening, grid=grid, max_time=max_time, precision=precision)
        self.calls = []
        Recorder.made.append(self)

    def init_gpu(self):
        self.calls.append("init_gpu")

    def init_benchmark(self):
        self.calls.append("init_benchmark")

    def run(self):
        self.calls.append("run")

    def single_run(self, *block):
        self.calls.append(("single_run", block))

    def print_results(self):
        self.calls.append("print")


@pytest.fixture
def recorder(monkeypatch):
    Recorder.made = []
    monkeypatch.setattr(B, "StencilBenchmark", Recorder)
    return Recorder


def test_2d_sweep_and_single_shape(recorder):
    base = ["bench", "Box", "2D", "1", "Jacobi", "Row", "None", "0", "1.0", "2", "2", "100", "90"]
    assert cli.main(base) == 0
    r = recorder.made[-1]
    assert r.args["grid"] == (100, 90, 1) and r.args["coarsening"] == (2, 2, 1) and r.args["dim"] == 2
    assert r.calls == ["init_gpu", "init_benchmark", "run", "print"]
    assert cli.main(base + ["32", "4"]) == 0
    assert recorder.made[-1].calls[2] == ("single_run", (32, 4, 1))


def test_3d_sweep_and_single_shape(recorder):
    base = ["bench", "Star", "3D", "2", "Variable", "Column", "Read", "16", "0.5", "1", "2", "4", "64", "65", "66"]
    assert cli.main(base) == 0
    r = recorder.made[-1]
    assert r.args["grid"] == (64, 65, 66) and r.args["coarsening"] == (1, 2, 4)
    assert r.args["align"] == "Read" and r.args["cl"] == 16 and r.args["max_time"] == 0.5
    assert r.calls[2] == "run"
    assert cli.main(base + ["8", "4", "2"]) == 0
    assert recorder.made[-1].calls[2] == ("single_run", (8, 4, 2))


def test_precision_option(recorder):
    argv = ["bench", "Box", "2D", "1", "Jacobi", "Row", "None", "0", "1.0", "1", "1", "64", "64", "--precision", "f32"]
    assert cli.main(argv) == 0
    assert recorder.made[-1].args["precision"] == "f32"


@pytest.mark.parametrize("argv", [
    ["bench", "Box", "2D", "1"],                                                                  # too few
    ["bench", "Box", "4D", "1", "Jacobi", "Row", "None", "0", "1.0", "2", "2", "100", "90"],      # dimension
    ["bench", "Box", "3D", "1", "Jacobi", "Row", "None", "0", "1.0", "2", "2", "100", "90"],      # 13 args in 3D
    ["bench", "Box", "2D", "one", "Jacobi", "Row", "None", "0", "1.0", "2", "2", "100", "90"],    # range
])
def test_bad_command_lines_print_the_usage(recorder, argv, capsys):
    assert cli.main(argv) == 1
    assert "Usage:" in capsys.readouterr().err
    assert not recorder.made


def test_results_tsv_matches_the_reference_report():
    b = B.StencilBenchmark("Star", 3, "Read", 16, "Variable", "Row", 2, (1, 2, 1), (40, 30, 20), 1.0)
    b.gpu_name = "NVIDIA B200"
    b.geom = b.spec.geometry(40, 30, 20)
    b.bench_results = [([0.5, 0.25], (32, 4, 2)), ([], (64, 1, 1))]
    lines = b.results_tsv().splitlines()
    e = b.geom.elements
    assert lines[0] == "#GPU: NVIDIA B200"
    assert lines[1] == "#grid size excluding border: x %d y %d z %d" % tuple(e[:3])
    assert lines[2] == "#coarsening factors: x 1 y 2 z 1"
    assert lines[3] == "#alignment: Read" and lines[4] == "#aligned to 128 byte"
    assert lines[5:10] == ["#orientation: Row", "#coefficients: Variable", "#neighbourhood: Star", "#range: 2",
                           "#dimension: 3"]
    assert lines[10].startswith("#xthreads\tythreads\tzthreads\tPerf [Flop/s]")
    assert len(lines) == 12  # a shape without durations is left out
    pts = float(b.geom.interior_points)
    lups = [pts / 0.5, pts / 0.25]
    mean = sum(lups) / 2
    sd = math.sqrt(sum((v - mean) ** 2 for v in lups) / 2)
    f = 2 * b.spec.stencil_size - 1  # Variable: 2S - 1 flops per update
    cols = lines[11].split("\t")
    assert cols[:3] == ["32", "4", "2"]
    assert float(cols[3]) == pytest.approx(mean * f, rel=1e-6)
    assert float(cols[4]) == pytest.approx(sd * f, rel=1e-6)
    assert float(cols[5]) == pytest.approx(mean, rel=1e-6) and float(cols[6]) == pytest.approx(sd, rel=1e-6)
    assert cols[7] == "2" and float(cols[8]) == pytest.approx(0.75)


def test_results_tsv_2d_rows():
    """2D: the z column reads 0, there is no alignment-size line, Jacobi counts S flops per update."""
    b = B.StencilBenchmark("Box", 2, "None", 0, "Jacobi", "Column", 1, (2, 2), (66, 34), 1.0)
    b.gpu_name = "g"
    b.geom = b.spec.geometry(66, 34)
    b.bench_results = [([1e-3], (128, 1, 1))]
    lines = b.results_tsv().splitlines()
    assert lines[1] == "#grid size excluding border: x 64 y 32" and lines[2] == "#coarsening factors: x 2 y 2"
    assert "#aligned to" not in "\n".join(lines)
    cols = lines[-1].split("\t")
    assert cols[:3] == ["128", "1", "0"]
    lups = 64 * 32 / 1e-3
    assert float(cols[5]) == pytest.approx(lups, rel=1e-6) and float(cols[3]) == pytest.approx(9 * lups, rel=1e-6)
    assert float(cols[6]) == 0.0 and cols[7] == "1"
