"""Dataset text files and the build plan (the reference's loadFromFile,
src/Data_Structures/File.cu:8-50, and adjustBuildPlan, src/core/QueryHandler.cu:23-45), on the CPU
through the C ABI's native reader."""
import numpy as np
import pytest


def test_reads_rows_and_ignores_extra_values(tb, tmp_path):
    X = np.random.default_rng(0).normal(0, 1, (50, 4))
    p = tmp_path / "demo_points.txt"
    with open(p, "w") as f:
        f.write("50 4\n")
        for r in X:
            f.write(" ".join("%.17g" % v for v in r) + " 123\n")  # a value past D is ignored
        f.write("trailing lines after row N are not read\n")
    Y = tb.load_dataset_file(str(p))
    assert Y.shape == (50, 4) and np.array_equal(X, Y)
    assert tb.extract_dataset_name(str(p)) == "demo"


@pytest.mark.parametrize("text,msg", [
    ("", "loadFromFile: empty file"),
    ("0 3\n", "loadFromFile: invalid header"),
    ("x 3\n", "loadFromFile: invalid header"),
    ("2 3\n1 2 3\n1 2\n", "loadFromFile: dimension mismatch at row 2"),
    ("2 3\n1 2 3\n1 2 x\n", "loadFromFile: dimension mismatch at row 2"),
    ("3 2\n1 2\n3 4\n", "loadFromFile: row count mismatch"),
])
def test_malformed_files(tb, tmp_path, text, msg):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    with pytest.raises(tb.TblaeqError) as e:
        tb.load_dataset_file(str(p))
    assert msg in str(e.value)
    with pytest.raises(tb.TblaeqError, match="cannot open"):
        tb.load_dataset_file(str(tmp_path / "missing.txt"))


def test_build_plan_truncation(tb):
    assert tb.adjust_build_plan(10_000_000, 4, (100, 50, 20)) == (4, [100, 50, 20])
    # The level that reaches a single centroid is kept; the levels above it are dropped.
    assert tb.adjust_build_plan(30_000, 4, (100, 50, 20)) == (4, [100, 50, 20])  # 300, 6, then 1
    assert tb.adjust_build_plan(1_000, 4, (100, 50, 20)) == (3, [100, 50])       # 10, then 1: 20 dropped
    assert tb.adjust_build_plan(50, 3, (100, 2)) == (2, [100])
    with pytest.raises(ValueError):
        tb.adjust_build_plan(100, 1, ())
    with pytest.raises(ValueError):
        tb.adjust_build_plan(100, 4, (10, 10))
