"""CPU checks of the synthetic input generators in bench.py (no GPU)."""
import numpy as np

import bench


def test_mt19937_64_matches_the_standard():
    # [rand.predef]: the 10000th output of a default-constructed std::mt19937_64 is 9981545732273789042
    assert int(bench.mt19937_64_stream(5489, 10000)[-1]) == 9981545732273789042
    g = bench.MT19937_64(4123)
    assert [g.next() for _ in range(700)] == [int(v) for v in bench.mt19937_64_stream(4123, 700)]


def test_batch_problem_recipe():
    sizes = [bench.batch_problem(p)[:2] for p in range(8)]
    assert all(32 <= nx <= 256 and 32 <= ny <= 256 for nx, ny in sizes)
    nx, ny, k = bench.batch_problem(0)
    assert k.shape == (nx * ny,) and np.all(k > 0)
    z = np.log(k)
    assert abs(z.mean()) < 0.05 and abs(z.std() - 1.0) < 0.05      # N(0, 1) conductivity exponents
    assert np.array_equal(k, bench.batch_problem(0)[2])               # deterministic


def test_sine_mode_initial_condition():
    A, B = bench.sine_modes(2)
    assert A.shape == (8, 3) and B.shape == (8,)
    assert np.all((A / np.pi >= 1) & (A / np.pi <= 8)) and np.all((B >= 0) & (B < 2 * np.pi))
