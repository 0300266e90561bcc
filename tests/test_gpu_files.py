"""bbt_fedsvd_run_files: the pipeline fed from the reference's on-disk input
(dpath/Client<c>.mat, dpath/y.mat; client.cpp:210-213, 1028) returns exactly
what the host-buffer entry returns on the same blocks, in both branches and in
svd_mode 4, and refuses missing or wrongly sized files before any work."""
import numpy as np
import pytest

import cases
import oracle
from excalibur_b200 import BBTError, datafiles
from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def same(a, b):
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, list):
        return all(np.array_equal(x, y) for x, y in zip(a, b))
    return np.array_equal(a, b)


@pytest.mark.parametrize("which", ["c1", "p3_uneven", "t_qr", "t_mixed", "t_qr_lr", "sq80"])
@pytest.mark.parametrize("precision", [0, 1])
def test_files_equal_host_entry(ctx, tmp_path, which, precision):
    y, mode, tall = None, 1, False
    if which in cases.pipeline_cases():
        blocks, seed = cases.pipeline_cases()[which]
    elif which == "sq80":
        blocks, seed = cases.square_cases()["sq80"]
    else:
        blocks, seed, y = cases.tall_cases()[which.replace("_lr", "")]
        tall = True
        if which.endswith("_lr"):
            mode = 4
        else:
            y = None
    datafiles.write_clients(str(tmp_path), blocks, y)
    m = blocks[0].shape[1] if tall else blocks[0].shape[0]
    ln = [b.shape[0] if tall else b.shape[1] for b in blocks]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s1, U1, V1 = ctx.fedsvd_files(str(tmp_path), m, ln, pub, priv, svd_mode=mode, precision=precision)
    s2, U2, V2 = ctx.fedsvd_host(blocks, pub, priv, svd_mode=mode, precision=precision, tall=tall, labels=y)
    assert same(s1, s2) and same(U1, U2) and same(V1, V2)


def test_files_large_tall_with_several_staging_chunks(ctx, tmp_path):
    """Blocks larger than one 64 MiB staging buffer (reads are split into
    chunks and over threads), split by the reference's own rule."""
    rng = np.random.default_rng(3)
    m, n, P = 120000, 300, 3   # 96 MB per file: two staging chunks each
    X = rng.standard_normal((m, n))
    blocks = datafiles.split_columns(X, P)
    datafiles.write_clients(str(tmp_path), blocks)
    ln = datafiles.partitions(n, P)
    pub, priv = oracle.reference_seeds(11, P)
    s1, U1, V1 = ctx.fedsvd_files(str(tmp_path), m, ln, pub, priv)
    s2, U2, V2 = ctx.fedsvd_host(blocks, pub, priv, tall=True)
    assert same(s1, s2) and same(U1, U2) and same(V1, V2)
    sl = np.linalg.svd(X, compute_uv=False)
    assert np.max(np.abs(s1 - sl) / sl) < 1e-11


def test_files_errors(ctx, tmp_path):
    blocks, seed = cases.pipeline_cases()["noqr"]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    m, ln = blocks[0].shape[0], [b.shape[1] for b in blocks]
    with pytest.raises(BBTError, match="BBT_ERR_IO.*Client0.mat"):
        ctx.fedsvd_files(str(tmp_path), m, ln, pub, priv)
    datafiles.write_clients(str(tmp_path), [blocks[0], blocks[1][:, :-1]])
    with pytest.raises(BBTError, match="BBT_ERR_IO.*Client1.mat holds"):
        ctx.fedsvd_files(str(tmp_path), m, ln, pub, priv)
    datafiles.write_clients(str(tmp_path), blocks)
    s, U, VT = ctx.fedsvd_files(str(tmp_path), m, ln, pub, priv)   # the context is still usable
    assert len(s) == m
