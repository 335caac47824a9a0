"""search_set restates the reference's SearchSet (inc/benchmarking/search_set.hpp:23-44):
std::mt19937 seeded 42 and std::uniform_int_distribution, random or a sequential
slice, one engine across repeats.  Pinned by the C++ standard's known answer for
mt19937 (the 10,000th output of a default-seeded engine is 4123659995) and by the
compiled reference's own SearchSet."""
import numpy as np
import pytest

from octrees_benchmark_b200.synth import MT19937, search_set


def test_mt19937_known_answer():
    g = MT19937(5489)
    assert int(g.next_u32(10_000)[-1]) == 4123659995


def test_mt19937_draws_in_pieces_equal_one_draw():
    a = MT19937(42).next_u32(2000)
    g = MT19937(42)
    b = np.concatenate([g.next_u32(7), g.next_u32(700), g.next_u32(1293)])
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n,cloud,seq", [(10, 100, False), (10_000, 1_000_000, False),
                                         (100_000, 10_000_000, False), (5_000, 3_000_000_000, False),
                                         (7, 7, False), (10, 100, True), (10_000, 1_000_000, True)])
def test_search_set_equals_the_reference(n, cloud, seq):
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref is not built")
    ref = oracle.Reference.search_set(n, cloud, sequential=seq, repeats=3).astype(np.int64)
    mine = np.stack([search_set(n, cloud, sequential=seq, repeat=r) for r in range(3)])
    assert np.array_equal(ref, mine)
