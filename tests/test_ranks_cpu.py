"""The bench's multi-rank plumbing on CPU: two gloo ranks (one process each,
as torchrun launches one per GPU) take the same barrier, agree on the max of
their times and report the whole-job rate from it."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    r, w, _ = bench.dist_env()
    bench.init_ranks(w, backend="gloo", timeout_s=60)
    bench.rank_barrier(w, cuda=False)
    ms = 100.0 + 50.0 * r  # rank 1 is the slow one
    mx = bench.max_over_ranks(ms, w, device="cpu")
    rate = bench.job_rate(10, w, mx)
    bench.close_ranks(w)
    q.put((r, mx, rate))


def test_two_gloo_ranks_agree_on_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for _, mx, rate in out:
        assert mx == 150.0
        assert abs(rate - 2 * 10 / 0.150) < 1e-9


def test_one_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_rate(10, 1, 100.0) == 100.0


def test_hbm_peak_names_its_source(tmp_path, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    v, src = bench.hbm_peak()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert "of measured" in src and v > 1000
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    v, src = bench.hbm_peak()
    assert v == 6650.0 and "of fallback" in src


def test_krylov_byte_model_matches_the_stated_formulas():
    """The roofline's algorithmic bytes per inner iteration, as stated with the
    kernels: mixed PCG (FP64 conjugate gradients, FP32 degree-16
    Chebyshev-Jacobi polynomial) reads 132 nnz + 456 N bytes (1370 B per row
    on the 524,288-cell channel); mixed BiCGStab-Jacobi 16 nnz + 104 N + 8."""
    sys.path.insert(0, ROOT)
    import bench
    N, nnz = 524288, 3629056
    def per(m, k=16):
        return (bench.krylov_bytes(N, nnz, 10, m, True, cheb_k=k) - bench.krylov_bytes(N, nnz, 0, m, True, cheb_k=k)) / 10
    assert per("pcg") == 132 * nnz + 456 * N
    assert round(per("pcg") / N) == 1370
    # degree k: one FP64 pass and k - 1 FP32 passes
    assert per("pcg", 24) == (12 + 8 * 23) * nnz + (96 + 24 * 23) * N
    assert per("bicg") == 16 * nnz + 104 * N + 8
