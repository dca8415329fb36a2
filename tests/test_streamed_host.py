"""Host logic of the out-of-core CP-ALS: the slab partition of the last mode."""
import pytest

import streamed


def test_slab_ranges_cover_the_mode_once():
    for extent in (1, 7, 30, 64, 513):
        for slab in (1, 3, 7, 64, 1000):
            r = streamed.slab_ranges(extent, slab)
            assert r[0][0] == 0 and r[-1][1] == extent
            assert all(b0 == a1 for (_, a1), (b0, _) in zip(r, r[1:]))
            assert all(0 < k1 - k0 <= slab for k0, k1 in r)


def test_slab_ranges_rejects_empty_slab():
    with pytest.raises(ValueError):
        streamed.slab_ranges(10, 0)
