"""Serving loop (rocblas_b200_server_*): continuous batching under an HBM budget, resident A /
invA reuse, and results that are bitwise the same alone and in the mix."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from rocblas_b200 import serving  # noqa: E402

pytestmark = pytest.mark.gpu

RESIDENT = {0: 200, 1: 700, 2: 1300, 3: 64, 4: 513, 5: 96}


def _server(budget=8 << 30, streams=2):
    srv = serving.TrsmServer(hbm_budget=budget, n_streams=streams, window_us=100.0,
                             keep_resident_copies=True)
    for key, m in RESIDENT.items():
        srv.add_resident(key, m, kband=key % 3 * 2, seed=10 + key)
    return srv


def _requests(n, rate, seed):
    return serving.make_requests(n, rate, seed, RESIDENT, m_range=(16, 1500), n_range=(1, 96))


def _oracle_check(srv, q, X):
    if q.a_key is not None:
        A = srv.residents[q.a_key].A[q.dtype].reshape(q.m, q.m)
    else:
        A = srv.payload_A(q)
    B = srv.payload_B(q)
    Ah = np.asfortranarray(np.tril(np.nan_to_num(A.cpu().numpy().T)))
    Bh = np.asfortranarray(B.cpu().numpy().T)
    ref = oracle.trsm("L", "L", "N", "N", 1.0, Ah, Bh)
    err = oracle.normwise_forward_error(X.cpu().numpy().T, ref)
    assert err < (1e-11 if q.dtype == "d" else 2e-3), (q.rid, q.m, q.n, q.dtype, err)


def test_serving_mix_equals_alone_and_is_correct():
    srv = _server()
    reqs = _requests(400, 20000.0, 3)
    lat = srv.run(reqs, keep_results=True)
    assert np.all(lat > 0)
    assert srv.last_stats["collections"] >= 1
    assert srv.last_stats["largest_collection"] > 1  # requests were batched
    mixed = {q.rid: q.B.clone() for q in reqs}
    for q in reqs[:40] + [q for q in reqs if q.m > 512][:10]:
        _oracle_check(srv, q, mixed[q.rid])
    srv.close()
    # the same requests one at a time through a fresh server: bitwise identical
    alone_srv = _server()
    for q in reqs[:60]:
        q2 = serving.Request(q.rid, 0.0, q.dtype, q.m, q.n, q.a_key, q.seed, q.kband)
        alone_srv.run([q2], keep_results=True)
        assert torch.equal(q2.B, mixed[q.rid]), (q.rid, q.m, q.n, q.dtype)
    alone_srv.close()


def test_serving_admission_respects_budget():
    srv = _server()
    base = srv.used
    reqs = _requests(200, 50000.0, 5)
    biggest = max(srv.request_bytes(q) for q in reqs)
    srv.set_budget(base + biggest + 1024)  # room for about one request at a time
    lat = srv.run(reqs)
    assert np.all(lat > 0)
    assert srv.last_stats["peak_bytes"] <= base + biggest + 1024
    assert srv.used == base
    srv.close()


def test_serving_rejects_bad_requests():
    srv = _server()
    q = serving.Request(0, 0.0, "d", 100, 4, 0, 1)  # resident 0 has m = 200, not 100
    with pytest.raises(serving.RocblasError):
        srv.run([q])
    srv.close()


def test_serving_host_payloads_equal_device_payloads():
    """Payloads read from pinned host memory across PCIe by the gather launch give the same
    results, bit for bit, as the same payloads in device memory."""
    reqs = _requests(120, 20000.0, 9)
    dev_srv = _server()
    dev_srv.run(reqs, keep_results=True)
    ref = {q.rid: q.B.clone() for q in reqs}
    dev_srv.close()
    host_srv = serving.TrsmServer(hbm_budget=8 << 30, n_streams=2, window_us=100.0,
                                  keep_resident_copies=True, payload_on_host=True)
    for key, m in RESIDENT.items():
        host_srv.add_resident(key, m, kband=key % 3 * 2, seed=10 + key)
    assert not host_srv.pool["d"].is_cuda and host_srv.pool["d"].is_pinned()
    lat = host_srv.run(reqs, keep_results=True)
    assert np.all(lat > 0)
    for q in reqs:
        assert torch.equal(q.B, ref[q.rid]), (q.rid, q.m, q.n, q.dtype)
    host_srv.close()
