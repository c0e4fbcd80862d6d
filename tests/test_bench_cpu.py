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


def test_serve_cpu_baseline_covers_the_whole_stream(built):
    """The serve CPU leg and the reference arm share one function: every
    distinct order of the stream is factored once, and the stream's CPU time
    weights those times by the counts of ALL the stream's requests (no request
    is skipped), so both report the same solves/s for the same stream."""
    for p in (str(ROOT), str(ROOT / "delayed-pivoting_b200"), str(ROOT / "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import bench
    from delayed_pivoting import serving as sv

    reqs = sv.make_stream(40, 5, hi=256)
    out = bench._cpu_serve_baseline(reqs, 5, lapack=False)
    orders = sorted({q.n for q in reqs})
    assert out["requests"] == len(reqs)
    assert out["solves"] == sum(len(q.solves) for q in reqs)
    assert sorted(int(k) for k in out["per_order_s"]) == orders
    expect = sum(out["per_order_s"][str(q.n)] for q in reqs)
    assert abs(out["stream_cpu_s"] - expect) <= 1e-3 * expect + 1e-4
    assert out["value"] > 0 and out["cores"] >= 1
    part = bench._cpu_serve_baseline(reqs, 5, orders=orders[:2], lapack=False)
    assert part["requests"] == sum(1 for q in reqs if q.n in orders[:2])
