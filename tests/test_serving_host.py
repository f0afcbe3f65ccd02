"""Host-side scheduler pieces of the serving engine (no GPU): the interval
allocator that places systems in the atom, pair and Green's-function pools."""
import numpy as np

from admp_b200.serving import _Intervals


def _model_free(cap, used):
    """Free runs of [0, cap) given the allocated (off, n) blocks."""
    occ = np.zeros(cap, bool)
    for off, n in used:
        occ[off:off + n] = True
    runs, k = [], 0
    while k < cap:
        if occ[k]:
            k += 1
            continue
        j = k
        while j < cap and not occ[j]:
            j += 1
        runs.append((k, j))
        k = j
    return runs


def test_intervals_random_alloc_release_against_model():
    rng = np.random.default_rng(3)
    for align in (1, 32):
        cap = 4096
        iv = _Intervals(cap, align)
        live = []
        for step in range(3000):
            if live and (rng.random() < 0.45 or len(live) > 60):
                off, n = live.pop(int(rng.integers(len(live))))
                iv.release(off, n)
            else:
                n = int(rng.integers(1, 200))
                off = iv.alloc(n)
                na = (n + align - 1) // align * align
                if off is not None:
                    assert off % align == 0 and off + na <= cap
                    assert all(off + na <= o or o + ((m + align - 1) // align * align) <= off for o, m in live)
                    live.append((off, n))
            used = [(o, (m + align - 1) // align * align) for o, m in live]
            assert iv.free == _model_free(cap, used)
            assert iv.used() == sum(n for _, n in used)


def test_intervals_first_fit_and_full_merge():
    iv = _Intervals(100)
    offs = [iv.alloc(10) for _ in range(10)]
    assert offs == list(range(0, 100, 10)) and iv.alloc(1) is None
    for o in (30, 50, 40):  # middle block freed last merges both sides
        iv.release(o, 10)
    assert iv.free == [(30, 60)]
    assert iv.alloc(25) == 30
    for o in offs:
        if not 30 <= o < 60:
            iv.release(o, 10)
    iv.release(30, 25)
    assert iv.free == [(0, 100)]
