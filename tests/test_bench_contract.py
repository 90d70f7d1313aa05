"""The benchmark's roofline bookkeeping (CPU only): the algorithmic-bytes
model and the DRAM traffic figure, which must come from an ncu capture of
the kernel sources as they are committed."""
import os
import sys

from conftest import REPO

sys.path.insert(0, REPO)


def test_algorithmic_bytes_model():
    """128 B per EGA evaluation (4 corners x 2 lookups x a bracketing pair
    of (u, eps) floats), 8 B Planck bracket per (point, channel), 16 + 8 G
    B per LOS point, 8 B per (ray, channel) out."""
    import bench
    assert bench.algorithmic_bytes(10, 3, 2, 4, 8) == 128 * 10 + 8 * 3 * 4 + (16 + 64) * 3 + 8 * 2 * 4
    assert bench.algorithmic_bytes(0, 0, 0, 64, 8) == 0


def test_kernel_families_cover_every_variant():
    import bench
    fams = [bench.kernel_family(v) for v in range(21)]
    assert fams[:9] == ["thread"] * 9 and fams[9:14] == ["lane"] * 5 and fams[14:] == ["ray"] * 7


def test_traffic_capture_matches_committed_kernel_sources():
    """Every captured traffic figure names the digest of the sources it was
    taken with; the committed figures describe the committed kernels."""
    import bench
    assert bench.TRAFFIC_PER_EGA
    for variant, (per_ega, sha) in bench.TRAFFIC_PER_EGA.items():
        assert 0 < per_ega < 128, variant  # below the algorithmic 128 B per evaluation
        assert sha == bench.kernel_sources_sha(bench.kernel_family(variant)), variant
        assert bench.dram_traffic(variant, 1000) == per_ega * 1000


def test_traffic_is_null_for_changed_sources_or_uncaptured_variants(monkeypatch):
    import bench
    assert bench.dram_traffic(6, 1000) is None
    v = next(iter(bench.TRAFFIC_PER_EGA))
    monkeypatch.setattr(bench, "kernel_sources_sha", lambda fam: "0" * 16)
    assert bench.dram_traffic(v, 1000) is None


def test_kernel_sources_exist():
    import bench
    for files in bench.KERNEL_SOURCES.values():
        for f in files:
            assert os.path.exists(os.path.join(REPO, "jurassic-scatter_b200", "csrc", f)), f
