"""The split of one job over several GPUs (dwcu_deconvolve_slabs): the
partition of z planes and z-pass columns among the parts (host arithmetic,
no device)."""
import pytest

import deconwolf_b200 as dw

SIZES = [
    ((60, 2048, 2048), (121, 193, 193)),  # job 2240 x 2240 x 180
    ((9, 22, 19), (5, 7, 9)),
    ((3, 30, 31), (5, 7, 9)),
    ((40, 256, 256), (79, 127, 127)),
]


@pytest.mark.parametrize("shape,psf_shape", SIZES)
@pytest.mark.parametrize("parts", [1, 2, 3, 4, 7, 8])
def test_every_plane_and_column_has_one_part(shape, psf_shape, parts):
    lay = [dw.slab_layout(shape, psf_shape, parts, p) for p in range(parts)]
    Z, cols, P = lay[0]["Z"], lay[0]["plane_cols"], shape[0]
    if parts > Z:
        pytest.skip("more parts than planes")
    # planes z = l*parts + p: the counts of a round-robin deal
    assert [q["planes"] for q in lay] == [len(range(p, Z, parts)) for p in range(parts)]
    assert [q["image_planes"] for q in lay] == [len(range(p, P, parts)) for p in range(parts)]
    assert sum(q["planes"] for q in lay) == Z and sum(q["image_planes"] for q in lay) == P
    assert max(q["planes"] for q in lay) - min(q["planes"] for q in lay) <= 1
    # z-pass columns: consecutive runs of whole kx blocks (multiples of 4)
    c = 0
    for q in lay:
        assert q["col0"] == c and q["col0"] % 4 == 0 and q["cols"] % 4 == 0 and q["cols"] > 0
        c += q["cols"]
    assert c == cols
    assert max(q["cols"] for q in lay) - min(q["cols"] for q in lay) <= 4


def test_bad_part_is_refused():
    with pytest.raises(dw.DwcuError):
        dw.slab_layout((9, 22, 19), (5, 7, 9), 2, 2)
    with pytest.raises(dw.DwcuError):
        dw.slab_layout((9, 22, 19), (5, 7, 9), 0, 0)
