"""The reference's text format (save_region_task.cc:37-67) through the C ABI,
no GPU needed: values printed with 20 significant digits and a tab each, one
row per line, blocks appended, an optional seed line per block; read back
whitespace-separated, row by row (direct_solve.cc:201-213)."""
import numpy as np
import pytest


def _reference_text(X, seed=None):
    # the format as save_data writes it: operator<< with setprecision(20)
    # is "%.20g"; a tab after every value, a newline after every row
    out = "" if seed is None else f"{seed}\n"
    for row in np.atleast_2d(X):
        out += "".join(f"{v:.20g}\t" for v in row) + "\n"
    return out


def test_write_matches_reference_format_and_reads_back(fs, tmp_path):
    rng = np.random.default_rng(3)
    X = rng.standard_normal((37, 5)) * 10.0 ** rng.integers(-300, 300, size=(37, 5))
    X[0, 0] = 0.0
    X[1, 1] = -0.0
    X[2, 2] = 1.0 / 3.0
    fn = str(tmp_path / "soln.txt")
    fs.write_text(fn, X)
    assert open(fn).read() == _reference_text(X)
    Y, seeds = fs.read_text(fn, 37, 5)
    assert seeds == []
    np.testing.assert_array_equal(Y, X)      # 20 digits round-trip every double


def test_blocks_with_seed_lines(fs, tmp_path):
    rng = np.random.default_rng(4)
    X = rng.standard_normal((30, 3))
    fn = str(tmp_path / "rhs.txt")
    blocks = [(0, 7), (7, 11), (18, 12)]
    for b, (r0, n) in enumerate(blocks):
        fs.write_text(fn, X[r0:r0 + n], seed=1245667 + b, print_seed=True)
    assert open(fn).read() == "".join(_reference_text(X[r0:r0 + n], 1245667 + b)
                                      for b, (r0, n) in enumerate(blocks))
    Y, seeds = fs.read_text(fn, 30, 3, block_rows=[n for _, n in blocks])
    np.testing.assert_array_equal(Y, X)
    assert seeds == [1245667, 1245668, 1245669]


def test_column_range(fs, tmp_path):
    X = np.arange(24, dtype=np.float64).reshape(4, 6) + 0.5
    fn = str(tmp_path / "cols.txt")
    fs.write_text(fn, X, col_beg=2, ncol=3)
    Y, _ = fs.read_text(fn, 4, 3)
    np.testing.assert_array_equal(Y, X[:, 2:5])


def test_read_errors(fs, tmp_path):
    fn = str(tmp_path / "short.txt")
    fs.write_text(fn, np.ones((3, 2)))
    with pytest.raises(fs.HodlrError) as e:
        fs.read_text(fn, 4, 2)                     # too few values
    assert e.value.status == fs.ERR_IO
    with pytest.raises(fs.HodlrError) as e:
        fs.read_text(str(tmp_path / "missing.txt"), 1, 1)
    assert e.value.status == fs.ERR_IO
    bad = tmp_path / "bad.txt"
    bad.write_text("1.0\tx\t\n")
    with pytest.raises(fs.HodlrError) as e:
        fs.read_text(str(bad), 1, 2)
    assert e.value.status == fs.ERR_IO
    with pytest.raises(fs.HodlrError):
        fs.read_text(fn, 3, 2, block_rows=[1, 1])  # blocks must cover the rows
