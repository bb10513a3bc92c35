"""Host-side logic of the library and the bench, without a GPU: the shared library loads and
exports every symbol include/cufe_b200.h declares, argument checks fail cleanly, and the
bench's multi-rank aggregation works over gloo."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "cufe_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|void|long long|const char \*|void \*)\s*\*?\s*(\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import cufe_b200 as cf
    L = cf.lib()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", cf.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s$" % n, out, re.M), n


def test_drop_in_symbols_have_the_reference_names():
    names = header_functions()
    for n in ("rlwe_sife_setup_gpu", "rlwe_sife_encrypt_gpu", "rlwe_sife_keygen_gpu", "rlwe_sife_decrypt_gmp_gpu"):
        assert n in names


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-device error path")
def test_errors_without_device():
    import ctypes as C
    import cufe_b200 as cf
    L = cf.lib()
    h = C.c_void_p()
    assert L.cufe_create(C.byref(h), 4096, 784, 0) == -5
    assert b"no CUDA device" in L.cufe_last_error()
    r = C.c_void_p()
    assert L.cufe_ring_create(C.byref(r), 4096, 3, None, 0) == -5
    with pytest.raises(cf.CufeError) as e:
        cf.Context(256, 8)
    assert e.value.code == -5


def test_argument_checks_before_device_use():
    import ctypes as C
    import cufe_b200 as cf
    L = cf.lib()
    h = C.c_void_p()
    assert L.cufe_create(None, 4096, 784, 0) == -1
    assert L.cufe_create(C.byref(h), 4095, 784, 0) == -1       # not a power of two
    assert L.cufe_create(C.byref(h), 16384, 784, 0) == -1      # above 8192
    assert L.cufe_create(C.byref(h), 4096, 0, 0) == -1         # empty vector
    assert L.cufe_ring_create(C.byref(h), 4096, 7, None, 0) == -1  # k above 6
    bad = np.array([16760831, 2147352577, 2130706433], np.uint32)  # not 1 mod 2n
    assert L.cufe_ring_create(C.byref(h), 4096, 3, bad.ctypes.data, 0) == -1
    for fn, args in (("cufe_sync", [None, None]), ("cufe_encrypt", [None, 1, None, None, None, None, None, None]),
                     ("cufe_decode", [None, 1, None, 1, None, None])):
        assert getattr(L, fn)(*args) == -1
    # drop-in with repeat < 1 reports through cufe_dropin_status without touching a device
    L.rlwe_sife_keygen_gpu(None, None, None, 0, None)
    assert L.cufe_dropin_status() == -1


def test_server_refuses_sizes_that_never_fit():
    """a tenant whose single encryption does not fit an empty tick (or whose ciphertext does not
    fit the arena) is refused at create, before any device is touched; so is a tick_bytes below
    the 1 MiB the server keeps for itself"""
    import ctypes as C
    import cufe_b200 as cf
    L = cf.lib()
    h = C.c_void_p()
    n = np.array([4096], np.int32)
    l = np.array([784], np.int32)

    def create(arena, tick, nn=n, ll=l):
        return L.cufe_server_create(C.byref(h), len(nn), nn.ctypes.data, ll.ctypes.data, arena, tick, 0)

    assert create(0, 1 << 19) == -1                     # below the server's own 1 MiB
    assert b"tick_bytes or arena_bytes is too small" in L.cufe_last_error()
    assert create(0, 64 << 20) == -1                    # one l = 784 encryption needs ~140 MB
    assert create(32 << 20, 0) == -1                    # a 38.6 MB ciphertext in a 32 MiB arena
    assert create(0, 0, np.array([4096, 3000], np.int32), np.array([8, 8], np.int32)) == -1
    if _no_gpu():                                       # sizes that fit reach the device check
        assert create(0, 1 << 30) == -5 and create(64 << 20, 256 << 20, ll=np.array([16], np.int32)) == -5


def test_sampler_refill_sizing():
    import cufe_b200 as cf
    L = cf.lib()
    # the precomputed refill range must cover the expected need with a wide margin:
    # mean accepted candidates per refill are 5.44 / 4.39 / 3.09 for S1 / S2 / S3
    for sig, mean in ((0, 5.44), (1, 4.39), (2, 3.09)):
        for calls, n in ((1, 256), (2, 4096), (784, 4096), (124, 2048)):
            R = L.cufe_sampler_refills(sig, calls, n)
            need = calls * (n / mean + 0.5)
            sd = (calls * n / mean) ** 0.5 * 1.4 / mean
            assert R >= need + 8 * sd, (sig, calls, n, R, need)
    assert L.cufe_sampler_refills(3, 1, 4096) == -1


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    ms_local = 100.0 + 50.0 * rank
    ms = bench.max_over_ranks(ms_local, "cpu")
    q.put((rank, ms))
    dist.destroy_process_group()


def test_bench_max_over_ranks_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res == {0: 150.0, 1: 150.0}
