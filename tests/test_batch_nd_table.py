"""Host-side table of the batched nD entry (lifted_image_t): packed offsets,
per-image and per-axis levels, wavelet names, and the argument errors."""
import pytest

from lifted_b200.batch import image_table


def test_packed_offsets_and_levels():
    tab, n = image_table([(4, 8), (2, 3, 5), (7,)], ["db2", 4, "cdf9.7"], [1, (2, 1, 0), 3])
    assert n == 3
    assert [tab[i].in_offset for i in range(3)] == [0, 32, 62]
    assert [tab[i].out_offset for i in range(3)] == [0, 32, 62]
    assert [tab[i].ndim for i in range(3)] == [2, 3, 1]
    assert list(tab[1].shape)[:3] == [2, 3, 5]
    assert list(tab[0].levels)[:2] == [1, 1] and list(tab[1].levels)[:3] == [2, 1, 0]
    assert tab[1].wavelet == 4 and tab[2].wavelet == 100907


def test_bad_tables():
    with pytest.raises(ValueError):
        image_table([(1, 2, 3, 4, 5)], "db2", 1)
    with pytest.raises(ValueError):
        image_table([(4, 4)], "db2", [(1, 2, 3)])
    with pytest.raises(ValueError):
        image_table([(4, 4), (4, 4)], ["db2"], 1)
