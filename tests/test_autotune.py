"""Host logic of the autotuner (no GPU): the candidate sets it may pick from and its cache
keys."""
from hindemith_b200 import autotune


def test_segment_candidates_respect_the_depth_and_the_image():
    """A candidate segment is the library default (0) or holds at least 2T rows (the
    temporal halo's lead-in) and fewer rows than the image."""
    for H in (1, 7, 16, 130, 512, 1080, 4096):
        for T in autotune.T_CANDIDATES:
            segs = autotune._seg_candidates(H, 1920, T)
            assert segs[0] == 0
            assert all(2 * T <= s < H for s in segs[1:]), (H, T, segs)


def test_candidate_depths_are_the_kernels_depths():
    assert set(autotune.T_CANDIDATES) == set(range(1, 9))
    for T, rows, layout in autotune.BATCH_CANDIDATES:
        assert 1 <= T <= 8 and rows > 0 and layout in (1, 2)


def test_tuning_run_length_is_part_of_the_cache_key():
    """A tuning over the workload's own sweep count is cached apart from the default one, and
    the default key is the one earlier caches hold."""
    k0 = autotune._sweep_key("B200", 1080, 1920, 1920, True, autotune.DEFAULT_TUNING_SWEEPS)
    k5 = autotune._sweep_key("B200", 1080, 1920, 1920, True, 500)
    assert k0 == "B200|1080x1920|ld1920|fast|layout"
    assert k5 != k0 and k5.startswith(k0)
    assert autotune._sweep_key("B200", 1080, 1920, 1920, False, 500) != k5
