"""The algorithmic byte counts behind the bench line's roofline fractions, at
128^3 (one species WhiteBearII + one cut-LJ interaction): the fused path's
per-stage count and the unfused 25-transform decomposition, mixed (4-byte
transforms) and FP64."""
import bench

N, NK = 128 ** 3, 128 * 128 * 65


def test_unfused_decomposition_bytes():
    assert bench.unfused_bytes(N, NK, 4) == 933_560_320
    assert bench.unfused_bytes(N, NK, 8) == 1_766_457_344
    # 445 bytes a point mixed, 842 FP64
    assert round(bench.unfused_bytes(N, NK, 4) / N) == 445
    assert round(bench.unfused_bytes(N, NK, 8) / N) == 842


def test_fused_stage_bytes():
    info = {"N": N, "Nk": NK, "channels": 11, "deriv_channels": 10, "precision": 1}
    st = bench.stage_bytes(info, fused=True)
    assert st["pointwise"] == 209_715_200
    assert bench.algorithmic_bytes(info, fused=True) == 832_372_736
    # fusing the passes removes ~11% of the unfused decomposition's bytes
    assert bench.algorithmic_bytes(info, fused=True) < bench.unfused_bytes(N, NK, 4)
