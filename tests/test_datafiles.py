"""The reference's on-disk input format (generate_data.cpp:19-45,
client.cpp:210-213, 549, 1028) as written and read by
excalibur_b200.datafiles.  CPU only."""
import numpy as np

from excalibur_b200 import datafiles as df


def test_partitions_rule():
    # n / P, the first n % P participants one more (generate_data.cpp:19-25)
    assert df.partitions(10, 3) == [4, 3, 3]
    assert df.partitions(9, 3) == [3, 3, 3]
    assert df.partitions(1000, 7) == [143] * 6 + [142]
    assert sum(df.partitions(12345, 64)) == 12345


def test_short_and_wide_layout_is_row_major_m_by_local_n():
    X = np.arange(4 * 10, dtype=np.float64).reshape(4, 10)
    blocks = df.split_columns(X, 3)
    assert [b.shape for b in blocks] == [(4, 4), (4, 3), (4, 3)]
    # xx[j + row * local_n] = X[row, counter + j] (generate_data.cpp:36)
    for b, o in zip(blocks, (0, 4, 7)):
        flat = b.ravel()
        for row in range(4):
            for j in range(b.shape[1]):
                assert flat[j + row * b.shape[1]] == X[row, o + j]


def test_tall_layout_is_column_major_m_by_local_n():
    X = np.arange(20 * 5, dtype=np.float64).reshape(20, 5)
    blocks = df.split_columns(X, 2)
    assert [b.shape for b in blocks] == [(3, 20), (2, 20)]
    # xx[j * m + row] = X[row, counter + j] (generate_data.cpp:35)
    for b, o in zip(blocks, (0, 3)):
        flat = b.ravel()
        for j in range(b.shape[0]):
            for row in range(20):
                assert flat[j * 20 + row] == X[row, o + j]


def test_lr_appends_a_bias_column_to_the_last_participant():
    X = np.random.default_rng(0).standard_normal((50, 7))
    blocks = df.split_columns(X, 3, lr=True)
    assert [b.shape[0] for b in blocks] == df.partitions(8, 3)
    assert np.all(blocks[-1][-1] == 1.0)          # tall: rows of X^T, the last is the bias
    assert np.array_equal(np.concatenate(blocks, axis=0)[:7], X.T)


def test_write_read_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    for m, n, P in ((30, 100, 3), (200, 40, 4)):
        X = rng.standard_normal((m, n))
        y = rng.standard_normal(m)
        blocks = df.split_columns(X, P)
        d = tmp_path / f"{m}x{n}"
        df.write_clients(str(d), blocks, y)
        tall = m > n
        for c, (b, w) in enumerate(zip(blocks, df.partitions(n, P))):
            assert (d / f"Client{c}.mat").stat().st_size == 8 * m * w
            assert np.array_equal(df.read_client(str(d), c, m, w, tall), b)
        assert np.array_equal(np.fromfile(d / "y.mat"), y)
