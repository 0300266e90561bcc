"""The reference's on-disk input format (Excalibur generate_data.cpp:19-45,
client.cpp:210-213, 1028): participant c of P reads dpath/Client<c>.mat,
raw float64 with no header, and in svd_mode 4 the last participant reads the
labels from dpath/y.mat (m values).

The features (columns) of X (m x n) are split over the participants as
n / P + (c < n % P) each.  A block is stored row-major m x local_n when
m <= n, and transposed (local_n x m row-major, i.e. column-major m x local_n)
when m > n, which is the layout run() reads in its tall-and-skinny branch
(client.cpp:549).  For linear regression the generator appends a column of
ones (the bias) to the last participant's block, so the partition is of n + 1
columns (generate_data.cpp:28, 39-42).

    blocks = split_columns(X, P)               # the reference's layout
    write_clients(dpath, blocks, y)             # Client<c>.mat (+ y.mat)
    ctx.fedsvd_files(dpath, m, [local_n...], public_seed, private_seeds)
"""
import os

import numpy as np

__all__ = ["partitions", "split_columns", "write_clients", "read_client"]


def partitions(n, P):
    """Columns per participant (generate_data.cpp:19-25)."""
    return [n // P + (1 if c < n % P else 0) for c in range(P)]


def split_columns(X, P, lr=False):
    """Participant blocks of X (m x n) in the reference's layout; with lr, a
    column of ones is appended before splitting (the bias term)."""
    X = np.asarray(X, dtype=np.float64)
    m = X.shape[0]
    if lr:
        X = np.concatenate([X, np.ones((m, 1))], axis=1)
    n = X.shape[1]
    tall = m > n
    out, o = [], 0
    for w in partitions(n, P):
        blk = X[:, o:o + w]
        out.append(np.ascontiguousarray(blk.T if tall else blk))
        o += w
    return out


def write_clients(dpath, blocks, y=None):
    """Write Client<c>.mat for each block as given (raw float64, C order)
    and y.mat when labels are given."""
    os.makedirs(dpath, exist_ok=True)
    for c, b in enumerate(blocks):
        np.ascontiguousarray(b, dtype=np.float64).tofile(os.path.join(dpath, f"Client{c}.mat"))
    if y is not None:
        np.ascontiguousarray(y, dtype=np.float64).tofile(os.path.join(dpath, "y.mat"))


def read_client(dpath, c, m, local_n, tall):
    """Participant c's block as run() sees it (m x local_n, or local_n x m
    when tall)."""
    x = np.fromfile(os.path.join(dpath, f"Client{c}.mat"), dtype=np.float64)
    if x.size != m * local_n:
        raise ValueError(f"Client{c}.mat holds {x.size} values, expected {m * local_n}")
    return x.reshape((local_n, m) if tall else (m, local_n))
