"""The CPU legs of bench.py (the reported CPU baselines), run without a GPU."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_cpu_baselines_time_the_reference_and_lapack(built):
    """The CPU legs of bench.py: the reference's delayed_getrf (or the oracle
    when the reference build is absent) and LAPACK dgetrf through the
    reference's wrapper, on the bench's own generator."""
    for p in (str(ROOT), str(ROOT / "delayed-pivoting_b200"), str(ROOT / "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import bench
    import oracle as orc

    g, t, kind, info = bench.cpu_reference_gflops(256, 16384, 1)
    assert g > 0 and t > 0 and info == 256
    assert kind == ("reference" if orc.ref_available() else "port")
    lap = bench.cpu_lapack_gflops(256, 16384, 1)
    if orc.ref_available():
        assert lap is not None and lap[0] > 0 and lap[1] > 0
    else:
        assert lap is None
