"""Host-side helpers of cumm.batch (CPU)."""
import torch

from cumm.batch import concat_clouds, lognormal_counts


def test_concat_clouds_sets_batch_and_offsets():
    a = torch.tensor([[0, 1, 2, 3], [0, 4, 5, 6]], dtype=torch.int32)
    b = torch.tensor([[0, 7, 8, 9]], dtype=torch.int32)
    c, offs = concat_clouds([a, b])
    assert offs == [0, 2, 3]
    assert c[:, 0].tolist() == [0, 0, 1]
    assert c[:, 1:].tolist() == [[1, 2, 3], [4, 5, 6], [7, 8, 9]]


def test_lognormal_counts_clipped_and_seeded():
    x = lognormal_counts(64, 40_000, 0.8, 5_000, 300_000, 0)
    assert len(x) == 64 and min(x) >= 5_000 and max(x) <= 300_000
    assert x == lognormal_counts(64, 40_000, 0.8, 5_000, 300_000, 0)
    assert 25_000 < sorted(x)[32] < 60_000
