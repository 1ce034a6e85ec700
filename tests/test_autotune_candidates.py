"""The autotuner's candidate launch shapes (host logic, no GPU): every
pipeline the library instantiates, FP64 limited to the shapes its kernels
have, and the four-cells-per-lane pipeline 4 offered to both sweep families
in FP32 only."""
from xlb_biot_b200 import autotune


def test_candidates_cover_every_pipeline_in_fp32():
    for kernel in (autotune.ELASTICITY, autotune.DARCY):
        pipes = {c["pipeline"] for c in autotune.candidates(4, kernel=kernel)}
        assert pipes == {0, 1, 2, 3, 4}, kernel


def test_fp64_candidates_skip_wide_tiles_and_pipeline_4():
    for kernel in (autotune.ELASTICITY, autotune.DARCY):
        cands = autotune.candidates(8, kernel=kernel)
        assert cands and all(c["tx"] == 128 and c["depth"] <= 4 and c["pipeline"] != 4 for c in cands)


def test_push_pipelines_vary_only_the_tile_width():
    for c in autotune.candidates(4):
        if c["pipeline"] in (3, 4):
            assert (c["depth"], c["ctas_per_sm"], c["min_rows"]) == (1, 1, 8)
    assert len({(c["tx"], c["depth"], c["ctas_per_sm"], c["min_rows"], c["pipeline"])
                for c in autotune.candidates(4)}) == len(autotune.candidates(4))
