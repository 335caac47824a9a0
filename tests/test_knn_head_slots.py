"""Group kNN head bookkeeping (CPU restatement of k_knn_group's index math).

Every kKnnHeadStride-th group (S = 16) is a head handed out first; slot s of
the other groups is group s + s / (S - 1) + 1.  This test checks that the
slots enumerate exactly the non-head groups, ascending, for every launch size
up to a few thousand groups, and that a group's seed head is the nearest head
of its own request (or none)."""
import pytest

S = 16  # kKnnHeadStride in cloud.h


def kernel_stride():
    import os
    import re
    src = open(os.path.join(os.path.dirname(__file__), "..", "octrees_benchmark_b200", "csrc", "cloud.h")).read()
    return int(re.search(r"kKnnHeadStride = (\d+);", src).group(1))


def test_stride_matches_source():
    assert kernel_stride() == S


@pytest.mark.parametrize("packets", list(range(0, 70)) + [255, 256, 257, 1000, 4096, 4097])
def test_slots_enumerate_the_non_heads(packets):
    n_heads = (packets + S - 1) // S
    slots = packets - n_heads
    groups = [s + s // (S - 1) + 1 for s in range(slots)]
    assert groups == [g for g in range(packets) if g % S != 0]
    assert [h * S for h in range(n_heads)] == [g for g in range(packets) if g % S == 0]


def seed_head(packet, pb, pe, n_heads):
    """The head k_knn_group reads for a run's first group (None: the density estimate)."""
    hlo = packet // S
    hhi = hlo + 1
    lo_ok = hlo * S >= pb
    hi_ok = hhi < n_heads and hhi * S < pe
    use_hi = hi_ok and (not lo_ok or hhi * S - packet < packet - hlo * S)
    return (hhi if use_hi else hlo) if (use_hi or lo_ok) else None


def test_seed_head_is_the_nearest_of_the_request():
    # three requests of 37, 5 and 90 groups in one launch
    bounds = [(0, 37), (37, 42), (42, 132)]
    packets = 132
    n_heads = (packets + S - 1) // S
    for pb, pe in bounds:
        heads = [h for h in range(n_heads) if pb <= h * S < pe]
        for g in range(pb, pe):
            if g % S == 0:
                continue
            h = seed_head(g, pb, pe, n_heads)
            if not heads:
                assert h is None
                continue
            assert h in heads
            best = min(abs(x * S - g) for x in heads)
            assert abs(h * S - g) == best or abs(h * S - g) <= S  # a neighbouring head of the request
