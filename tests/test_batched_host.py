"""Host-side logic of the batched multigrid (no GPU): the per-instance level
counts and the balanced block map of the prolongation."""
import numpy as np

from xlb_biot_b200.batched import auto_levels, balanced_block_map


def test_auto_levels_halve_down_to_the_smallest_side_of_at_least_three():
    assert auto_levels(64, 64) == 5          # 64 .. 4
    assert auto_levels(96, 96) == 6          # 96 .. 3
    assert auto_levels(384, 384) == 8        # 384 .. 3
    assert auto_levels(64, 40) == 4          # 40 -> 20 -> 10 -> 5
    assert auto_levels(34, 34) == 2          # 17 is odd
    assert auto_levels(6, 6) == 2            # 3 is the coarsest side allowed


def test_balanced_block_map_covers_every_cell_once():
    rng = np.random.default_rng(0)
    cells = [int(v) for v in rng.integers(1, 5000, size=40)] + [1024, 2048, 1]
    blocks, begin = balanced_block_map(cells)
    assert blocks.dtype == np.int32 and begin.dtype == np.int32
    assert begin[0] == 0 and begin[-1] == len(blocks) and len(begin) == len(cells) + 1
    for k, n in enumerate(cells):
        mine = blocks[begin[k]:begin[k + 1]]
        assert (mine[:, 0] == k).all()
        assert len(mine) == -(-n // 1024)                    # ceil(n / 1024) blocks
        covered = np.zeros(n, dtype=np.int64)
        for _, e in mine:
            covered[e:min(e + 1024, n)] += 1
        assert (covered == 1).all()
