"""Host-side scheduler pieces of the serving engine (no GPU): the interval
allocator that places systems in the atom, pair and Green's-function pools,
the policy that decides which launched records the host waits for, the call
timeline accounting and the packing of request arrays into pool slices."""
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


class _Ev:
    """Stand-in for a CUDA event: `done` says whether the device passed it."""

    def __init__(self, done):
        self.done = done
        self.waited = False

    def query(self):
        return self.done

    def synchronize(self):
        self.waited = True
        self.done = True


class _Sched:
    """Just the state ServingEngine._drain reads and the completions it calls."""

    def __init__(self, recs):
        self._inflight = list(recs)
        self.host_time = {"wait": 0.0, "results": 0.0}
        self.completed = []

    def _complete_finish(self, rec, now_fn):
        self.completed.append(rec[2])

    def _complete_iterate(self, rec):
        self.completed.append(rec[2])


def test_drain_keeps_the_current_steps_records_in_flight():
    from admp_b200.serving import ServingEngine
    drain = ServingEngine._drain
    # no CG batch running: older records are waited for, the newest one (this step's) stays
    s = _Sched([("finish", _Ev(False), "a"), ("finish", _Ev(False), "b"), ("finish", _Ev(False), "c")])
    drain(s, None, 0, 1)
    assert s.completed == ["a", "b"] and [r[2] for r in s._inflight] == ["c"]
    # a record of this step whose event already passed completes without waiting
    s = _Sched([("finish", _Ev(False), "a"), ("finish", _Ev(True), "b")])
    drain(s, None, 0, 1)
    assert s.completed == ["a", "b"] and not s._inflight
    # a step that launched nothing waits for everything (no spinning on the host)
    s = _Sched([("finish", _Ev(False), "a"), ("finish", _Ev(False), "b")])
    drain(s, None, 0, 0)
    assert s.completed == ["a", "b"] and not s._inflight
    # CG batches running: the oldest records are waited for until one iterate record is
    # outstanding; records after that complete only once their events passed
    evs = [_Ev(False), _Ev(False), _Ev(False), _Ev(False)]
    s = _Sched([("iter", evs[0], "i1"), ("finish", evs[1], "f1"), ("iter", evs[2], "i2"), ("finish", evs[3], "f2")])
    drain(s, None, 1, 2)
    assert s.completed == ["i1"] and [r[2] for r in s._inflight] == ["f1", "i2", "f2"]
    assert evs[0].waited and not evs[1].waited and not evs[2].waited


class _TEv:
    """Stand-in for a timing CUDA event recorded at device time t (ms)."""

    def __init__(self, t):
        self.t = t

    def elapsed_time(self, other):
        return other.t - self.t


def test_call_timeline_accounts_spans_and_gaps():
    from admp_b200.serving import ServingEngine

    class _S:
        call_trace = [("nb", _TEv(2.0), _TEv(5.0)), ("ef", _TEv(5.0), _TEv(9.0)), ("nb", _TEv(12.5), _TEv(14.0))]

    tl = ServingEngine.call_timeline(_S(), _TEv(0.0), _TEv(15.0), top=2)
    assert tl["pass_ms"] == 15.0
    assert tl["calls"] == {"nb": {"n": 2, "ms": 4.5}, "ef": {"n": 1, "ms": 4.0}}
    assert tl["gap_ms"] == 2.0 + 0.0 + 3.5 + 1.0
    assert tl["largest_gaps"] == [{"ms": 3.5, "after": "ef", "before": "nb"},
                                  {"ms": 2.0, "after": "start", "before": "nb"}]


def test_fill_device_tensor_parts_with_padding():
    """_fill's tensor branch (what admission uses for device-resident requests), run on CPU tensors:
    every request array lands at its offset, reshaped to the pool's row width and converted to the
    pool's dtype, with zero rows in the alignment gaps."""
    import torch
    from admp_b200.serving import ServingEngine

    class _S:
        _zeros = {dt: torch.zeros(3 * 64, dtype=dt) for dt in (torch.float32, torch.float64)}
        _zero_views = {}

    rng = np.random.default_rng(5)
    for width, shapes in ((3, [(4, 3), (7, 3), (1, 3)]), (1, [(5,), (2,), (3,)]), (9, [(3, 3), (3, 3)])):
        for dt in (torch.float32, torch.float64):
            arrays = [torch.tensor(rng.standard_normal(sh), dtype=torch.float64) for sh in shapes]
            pads = [int(rng.integers(0, 4)) for _ in shapes[:-1]] + [0]
            rows = sum(a.numel() // width + p for a, p in zip(arrays, pads))
            dest = torch.full((rows * width,), float("nan"), dtype=dt)
            for _ in range(2):  # the second call reuses the cached padding views
                assert ServingEngine._fill(_S(), dest, arrays, pads, width) == 0
                ref = []
                for a, p in zip(arrays, pads):
                    ref.append(a.reshape(-1).to(dt))
                    ref.append(torch.zeros(p * width, dtype=dt))
                assert torch.equal(dest, torch.cat(ref))
