"""Shared helpers for the GPU tests (imported only by tests marked gpu)."""
import numpy as np
import pytest


def context():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import excalibur_b200 as eb
    return eb.Context(0)


def subspace_angle(A, B):
    """Largest principal angle between the column spaces of A and B, from
    the sine form ||(I - Qa Qa^T) Qb|| (accurate for tiny angles, unlike
    arccos of the cosines which bottoms out near 1.5e-8)."""
    import scipy.linalg
    return float(np.max(scipy.linalg.subspace_angles(A, B)))


def gap_groups(sigma, rel_gap=1e-6):
    """Split indices of a descending spectrum into groups separated by a
    relative gap > rel_gap (well-posed subspaces)."""
    groups, cur = [], [0]
    for i in range(1, len(sigma)):
        if (sigma[i - 1] - sigma[i]) > rel_gap * sigma[0]:
            groups.append(cur)
            cur = [i]
        else:
            cur.append(i)
    groups.append(cur)
    return groups
