#!/usr/bin/env python
"""bench.py -- IPFE inner products/sec at N=4096 (bit-exact), batched vs plain GPU; p99 ms.

Workload (the reference's plain GPU pipeline shape): ring N = 4096, the three params.h RNS
primes, l = 784 (p = 50177), x uniform in [0, 4], y uniform in [-16, 16], 10,000 encryptions
x 1 function key, seeded synthetic data (SplitMix-style numpy seeds).  One inner product =
encrypt(x) + keygen(y) (one key, done once) + decrypt + decode of all N coefficients; the
inner product is coefficient 0, centred.  A step is one batch of B encryptions through the
whole pipeline; the batch output is checked against the plaintext dot products after timing.

Besides the batched value the line carries: "plain" (one encryption per call, device-resident,
the same kernels), "plain_dropin" (the reference's per-call form through the four
rlwe_sife_*_gpu symbols on host buffers), "coef0" (batched with the constant-coefficient
decrypt), "e2e" (batched through the C ABI with pinned host inputs and results), the roofline
of the dominant kernel and the clocks sampled during the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl cufe|reference]

--impl reference times the reference's own CPU implementation (cuFE src/*.c compiled from
source, oracle/_ref) on this host's cores, one process per core.  Under torchrun each rank
drives its own GPU with an independent replica of the workload (the path has no exchange
step); the value is all ranks' inner products over the slowest rank's time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, L = 4096, 784
TOTAL_ENC = 10000
METRIC = "IPFE inner products/sec at N=4096 (bit-exact), batched vs plain GPU; p99 ms"
UNIT = "IP/s"
SEED = 0xC0FE0002


def workload():
    rng = np.random.default_rng(SEED)
    x = rng.integers(0, 5, (TOTAL_ENC, L), dtype=np.uint32)
    y = rng.integers(-16, 17, (1, L), dtype=np.int32)
    seeds2 = rng.integers(0, 256, (TOTAL_ENC, 32), dtype=np.uint8)
    seeds3 = rng.integers(0, 256, (TOTAL_ENC, 32), dtype=np.uint8)
    setup_seeds = rng.integers(0, 256, (3, 32), dtype=np.uint8)
    return x, y, seeds2, seeds3, setup_seeds


def max_over_ranks(value, device):
    """max of a per-rank float over the process group (identity without one)"""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ----------------------------------------------------------------------------- clocks

class Clocks:
    def __init__(self, device, out):
        self.out = out
        self.p = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(out, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        rows = []
        for line in open(self.out):
            f = [t.strip() for t in line.split(",")]
            if len(f) >= 7:
                try:
                    rows.append((float(f[0]), float(f[1]), f[3:7]))
                except ValueError:
                    pass
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- reference arm

def _ref_worker_init(path):
    global _REF, _REFDATA
    from oracle.ffi import Reference
    _REF = Reference("n4096_l784")
    d = np.load(path)
    _REFDATA = {k: d[k] for k in d.files}


def _ref_one(i):
    """one inner product on the reference CPU path: encrypt + two decrypts (signed y split
    into y+ - y-, since the reference reduces y as uint32) with their GMP decode"""
    d = _REFDATA
    ct = _REF.encrypt(d["x"][i], d["mpk"], d["s2"][i])
    _, dp = _REF.decrypt(ct, d["yp"], d["skp"])
    _, dm = _REF.decrypt(ct, d["ym"], d["skm"])
    p = 64 * L + 1

    def centred(v):
        v = int(v) % p
        return v - p if v > p // 2 else v
    return centred(int(dp[0]) - int(dm[0]))


def reference_pool(x, y, seeds2, setup_seeds, nproc):
    """spawned processes with the reference CPU build; keys made once by the reference setup"""
    import multiprocessing as mp
    from oracle.ffi import Reference
    R = Reference("n4096_l784")
    mpk, msk = R.setup(setup_seeds[0], setup_seeds[2])
    yv = y[0].astype(np.int64)
    yp = np.where(yv > 0, yv, 0).astype(np.uint32)
    ym = np.where(yv < 0, -yv, 0).astype(np.uint32)
    skp, skm = R.keygen(yp, msk), R.keygen(ym, msk)
    tmp = tempfile.NamedTemporaryFile(suffix=".npz", delete=False)
    np.savez(tmp.name, x=x, mpk=mpk, s2=seeds2, yp=yp, ym=ym, skp=skp, skm=skm)
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(nproc, initializer=_ref_worker_init, initargs=(tmp.name,))
    return pool, tmp.name


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    x, y, seeds2, _, setup_seeds = workload()
    nproc = max(1, min(os.cpu_count() or 1, args.ref_procs))
    pool, path = reference_pool(x, y, seeds2, setup_seeds, nproc)
    try:
        idx = 0
        times = []
        ok = True
        for step in range(args.warmup + args.steps):
            ids = [(idx + j) % TOTAL_ENC for j in range(nproc)]
            idx += nproc
            t0 = time.perf_counter()
            res = pool.map(_ref_one, ids)
            dt = time.perf_counter() - t0
            exp = [int(x[i].astype(np.int64) @ y[0].astype(np.int64)) for i in ids]
            ok = ok and res == exp
            if step >= args.warmup:
                times.append(dt)
    finally:
        pool.terminate()
        os.unlink(path)
    total = sum(times)
    value = nproc * len(times) / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint32",
            "data": "synthetic", "bit_exact": ok,
            "config": {"workload": "N=4096 l=784, x in [0,4], y in [-16,16], 10000 encryptions x 1 key",
                       "n": N, "l": L, "step": "%d inner products, one per process" % nproc},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference",
                             "sample": "%d steps x %d processes, 1 inner product each (encrypt + "
                                       "2 decrypts for signed y + GMP decode)" % (args.steps, nproc)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(x, y, seeds2, setup_seeds, nproc, steps=2):
    pool, path = reference_pool(x, y, seeds2, setup_seeds, nproc)
    try:
        pool.map(_ref_one, list(range(nproc)))  # warm
        t0 = time.perf_counter()
        for s in range(steps):
            pool.map(_ref_one, [(nproc * (s + 1) + j) % TOTAL_ENC for j in range(nproc)])
        dt = time.perf_counter() - t0
    finally:
        pool.terminate()
        os.unlink(path)
    return {"value": nproc * steps / dt, "unit": UNIT, "cores": nproc, "kind": "reference",
            "sample": "%d rounds x %d processes, 1 inner product each (reference CPU build, "
                      "encrypt + 2 decrypts for signed y + GMP decode)" % (steps, nproc)}


# ----------------------------------------------------------------------------- GPU arm

# DRAM bytes per refill of the sigma_3 candidate kernel, from one ncu capture of a batch-16
# launch (dram__bytes_read.sum + dram__bytes_write.sum = 1.23 MB + 530.3 MB over
# 16 x 1,044,352 refills: 31.8 B against 35 B algorithmic, because the last tens of MB that
# the launch writes are still in L2 when it ends); traffic grows with the refill count, so a
# launch of B streams moves B x refills x this
CAND_S3_DRAM_BYTES_PER_REFILL = (1.231872e6 + 530.28736e6) / (16 * 1044352)


# algorithmic HBM bytes per launch of each kernel at this workload (batch B)
def algorithmic_bytes(kernel, B, refills3):
    poly = 3 * N * 4
    return {
        "sample_cand_s3": refills3 * B * 35,           # 8 low words, accept mask, bit-32/sign bytes
        "sample_scatter": refills3 * B * 35 + B * L * poly,  # candidates and masks; f_i residues
        "encrypt_intt": (L + 1) * poly + B * (L * poly + (L + 1) * poly),  # mpk once, f_i, ciphertexts
        "decrypt_mac": B * (L + 1) * poly + B * poly,    # ciphertexts read, partial sums written
        "decode": B * poly + B * N * 4,
    }.get(kernel)


def crt_decode(v, p):
    """Garner CRT of one coefficient's three residues and the reference's rounding
    (crt_reverse_gmp + round_extract_gmp2, src/crt.c:46-81, src/rlwe_sife.c:334-393): the
    caller-side host decode of the drop-in form"""
    from cufe_b200 import Q
    q = Q[0] * Q[1] * Q[2]
    x = 0
    for j in range(3):
        mj = q // Q[j]
        x += int(v[j]) * mj * pow(mj, -1, Q[j])
    x %= q
    quo, rem = divmod(p * x, q)
    return quo + (1 if rem > q // 2 else 0)


def dropin_plain(cf, ctx, mpk, msk, x, y, seeds2, calls, device):
    """The reference's plain per-call GPU form: per inner product one rlwe_sife_encrypt_gpu
    (repeat 1) and one rlwe_sife_decrypt_gmp_gpu (two keys: y+ and y-, since the reference
    reduces y as uint32) on host buffers, synchronous, then the host decode of coefficient 0.
    Keys come from one rlwe_sife_keygen_gpu call made before timing."""
    import ctypes as C
    L_ = cf.lib()
    if L_.cufe_dropin_configure(N, L, device) != 0:
        return {"value": None, "error": "cufe_dropin_configure failed"}
    mpk_h = np.ascontiguousarray(cf.u32(mpk))
    msk_h = np.ascontiguousarray(cf.u32(msk))
    yv = y[0].astype(np.int64)
    ys = np.stack([np.where(yv > 0, yv, 0), np.where(yv < 0, -yv, 0)]).astype(np.uint32)
    sk = np.zeros((2, 3, N), np.uint32)
    L_.rlwe_sife_keygen_gpu(ys.ctypes.data, msk_h.ctypes.data, sk.ctypes.data, 2, None)
    ct = np.zeros((L + 1, 3, N), np.uint32)
    dy = np.zeros((2, 3, N), np.uint32)
    p = 64 * L + 1
    lat, ok = [], True
    for i in range(calls + 2):
        xi = np.ascontiguousarray(x[i])
        s2 = np.ascontiguousarray(seeds2[i])
        t0 = time.perf_counter()
        L_.rlwe_sife_encrypt_gpu(xi.ctypes.data, mpk_h.ctypes.data, ct.ctypes.data, s2.ctypes.data, s2.ctypes.data, 1,
                                 None)
        L_.rlwe_sife_decrypt_gmp_gpu(ct.ctypes.data, ys.ctypes.data, sk.ctypes.data, dy.ctypes.data, 2, None)
        v = (crt_decode(dy[0, :, 0], p) - crt_decode(dy[1, :, 0], p)) % p
        t1 = time.perf_counter()
        v = v - p if v > p // 2 else v
        ok = ok and v == int(x[i].astype(np.int64) @ yv)
        if i >= 2:
            lat.append(1000.0 * (t1 - t0))
    ok = ok and L_.cufe_dropin_status() == 0
    return {"value": 1000.0 * len(lat) / sum(lat), "unit": UNIT, "calls": len(lat),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)), "bit_exact": ok,
            "form": "reference per-call form: rlwe_sife_encrypt_gpu (repeat 1) + rlwe_sife_decrypt_gmp_gpu "
                    "(2 keys) on pageable host buffers, synchronous, host decode of coefficient 0; GPU counter "
                    "mapping; wall clock"}


def gpu_arm(args):
    import torch
    import cufe_b200 as cf
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = "cuda:%d" % local
    x, y, seeds2, seeds3, setup_seeds = workload()
    B = args.batch
    nb = TOTAL_ENC // B
    ctx = cf.Context(N, L, device=local)
    mpk, msk = ctx.setup(setup_seeds[0], setup_seeds[1], setup_seeds[2])
    y_dev = torch.from_numpy(y.copy()).to(dev)
    sky = ctx.keygen(y_dev, msk, y_signed=True)
    x_dev = cf.to_dev(x, dev)
    ct = ctx.ct_buf(B)
    dy = torch.empty((B, 1, 3, N), dtype=torch.int32, device=dev)
    steps, warm = args.steps, args.warmup
    res = torch.empty((steps, B, N), dtype=torch.int32, device=dev)
    scratch = torch.empty((B, N), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(local)

    def first(k):
        """first encryption of step k on this rank: ranks take disjoint batches"""
        return ((k * world + rank) % nb) * B

    def step(k, out):
        b0 = first(k)
        ctx.encrypt(x_dev[b0:b0 + B], mpk, seeds2[b0:b0 + B], seeds3[b0:b0 + B], ct=ct)
        ctx.decrypt(ct, y_dev, sky, y_signed=True, dy=dy)
        ctx.decode(dy, out=out)

    # the encryption shape for this batch size, chosen by the library's tuner (bit-exact either way)
    b0 = first(0)
    enc_group, enc_ms = ctx.tune_encrypt(x_dev[b0:b0 + B], mpk, seeds2[b0:b0 + B], seeds3[b0:b0 + B], ct=ct)
    for w in range(warm):
        step(w, scratch)
    ctx.sync()

    # --- batched, device-resident inputs (value)
    clk = Clocks(local, os.path.join(tempfile.gettempdir(), "cufe_clocks_%d.csv" % rank))
    ctx.profile_reset()
    ctx.profile(True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    e0.record(stream)
    step_ev[0].record(stream)
    for k in range(steps):
        step(warm + k, res[k])
        step_ev[k + 1].record(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.stop()
    ctx.profile(False)
    prof = ctx.profile_read()
    timed_launches = ctx.profile_launches()
    ctx.sync()
    step_ms = [step_ev[i].elapsed_time(step_ev[i + 1]) for i in range(steps)]
    ms = max_over_ranks(ms, dev)
    # correctness of every inner product in the timed region
    got = cf.u32(res[:, :, 0]).astype(np.int64)
    p = ctx.p
    got = np.where(got > p // 2, got - p, got)
    ids = np.array([first(warm + k) + j for k in range(steps) for j in range(B)]).reshape(steps, B)
    exp = x[ids].astype(np.int64) @ y[0].astype(np.int64)
    bit_exact = bool((got == exp).all())
    ips = steps * B * world / (ms / 1000.0)

    # --- plain per-call form: one encryption per call, synchronised each call
    nplain = args.plain_calls
    pl_ct = ctx.ct_buf(1)
    pl_dy = torch.empty((1, 1, 3, N), dtype=torch.int32, device=dev)
    pl_out = torch.empty((1, N), dtype=torch.int32, device=dev)
    lat = []
    for i in range(nplain + 2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.encrypt(x_dev[i:i + 1], mpk, seeds2[i:i + 1], seeds3[i:i + 1], ct=pl_ct)
        ctx.decrypt(pl_ct, y_dev, sky, y_signed=True, dy=pl_dy)
        ctx.decode(pl_dy, out=pl_out)
        b.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            lat.append(a.elapsed_time(b))
    plain = {"value": 1000.0 * len(lat) / sum(lat), "unit": UNIT, "calls": len(lat),
             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
             "form": "one encryption per call (batch 1), device-resident, same kernels"}
    # per-kernel device time of the plain form, from a few more calls profiled apart from the
    # timed ones (the per-launch events would add to the measured latency)
    ctx.profile_reset()
    ctx.profile(True)
    npr = 4
    for i in range(npr):
        ctx.encrypt(x_dev[i:i + 1], mpk, seeds2[i:i + 1], seeds3[i:i + 1], ct=pl_ct)
        ctx.decrypt(pl_ct, y_dev, sky, y_signed=True, dy=pl_dy)
        ctx.decode(pl_dy, out=pl_out)
        torch.cuda.synchronize()
    ctx.profile(False)
    plain_prof = ctx.profile_read()

    # --- batched with the constant-coefficient decrypt (decrypt + decode of coefficient 0 only)
    r0 = torch.empty((steps, B, 1), dtype=torch.int32, device=dev)
    c0_form, c0_tune_ms = ctx.tune_decrypt_coef0(ct, y_dev, sky, y_signed=True, out=r0[0])
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for k in range(steps):
        b0 = first(warm + k)
        ctx.encrypt(x_dev[b0:b0 + B], mpk, seeds2[b0:b0 + B], seeds3[b0:b0 + B], ct=ct)
        ctx.decrypt_coef0(ct, y_dev, sky, y_signed=True, out=r0[k])
    g1.record(stream)
    torch.cuda.synchronize()
    c0_ms = max_over_ranks(g0.elapsed_time(g1), dev)
    g = cf.u32(r0[:, :, 0]).astype(np.int64)
    coef0 = {"value": steps * B * world / (c0_ms / 1000.0), "unit": UNIT, "ms_per_step": c0_ms / steps,
             "bit_exact": bool((np.where(g > p // 2, g - p, g) == exp).all()),
             "form": "batched, decrypt and decode of coefficient 0 only (the coefficient the reference decodes)"}

    # --- the reference's plain per-call GPU form, through the drop-in symbols
    plain_dropin = dropin_plain(cf, ctx, mpk, msk, x, y, seeds2, args.dropin_calls, local)

    # --- end to end through the C ABI with host buffers (pinned), copies in the timed region
    xh = torch.from_numpy(x.view(np.int32)).pin_memory()
    rh = torch.empty((steps, B), dtype=torch.int32).pin_memory()
    xd = torch.empty((B, L), dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for k in range(steps):
        b0 = first(warm + k)
        xd.copy_(xh[b0:b0 + B], non_blocking=True)
        ctx.encrypt(xd, mpk, seeds2[b0:b0 + B], seeds3[b0:b0 + B], ct=ct)
        ctx.decrypt(ct, y_dev, sky, y_signed=True, dy=dy)
        ctx.decode(dy, out=scratch)
        rh[k].copy_(scratch[:, 0], non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_ok = bool((np.where(rh.numpy().view(np.uint32).astype(np.int64) > p // 2,
                            rh.numpy().view(np.uint32).astype(np.int64) - p,
                            rh.numpy().view(np.uint32).astype(np.int64)) == exp).all())
    e2e = {"value": steps * B * world / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": B * L * 4 + B * 64, "d2h_bytes_per_step": B * 4, "bit_exact": e2e_ok}

    # --- roofline of the dominant kernel (device time summed over the timed region)
    from cufe_b200 import _refills_s3
    refills3 = _refills_s3(N, L)
    launches = timed_launches
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    name, (cnt, tot) = dom
    per_launch_s = tot / cnt / 1000.0
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    abytes = algorithmic_bytes(name, B, refills3)
    roof = {"kernel": name, "bound": "hbm", "unit": "GB/s", "peak": hbm_peak,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "achieved": (abytes / per_launch_s / 1e9) if abytes else None,
            "traffic": (CAND_S3_DRAM_BYTES_PER_REFILL * refills3 * B) if name == "sample_cand_s3" else None,
            "algorithmic_bytes": abytes,
            "share": tot / sum(v[1] for v in prof.values())}
    roof["frac"] = roof["achieved"] / hbm_peak if roof["achieved"] else None
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0

    def lds_pipe(batch, launch_s):
        # the AES keystream bounds the sigma_3 candidate kernel: 13 AES-256 blocks per refill;
        # with the counter caching a block takes 1 + 4 + 11 x 16 + 16 = 197 T-table lookups from
        # shared memory, plus 15 per refill for the round-2 constants (one warp LDS per clock
        # per SM): 198 per block
        blocks = refills3 * batch * 13
        lds_peak = 148 * sm_mhz * 1e6 * 32 / 198
        return {"what": "AES-256 blocks/s (T-table, shared-memory LDS bound)", "achieved": blocks / launch_s,
                "peak_lds_bound": lds_peak, "frac": blocks / launch_s / lds_peak, "sm_mhz": sm_mhz}

    if name.startswith("sample_cand"):
        roof["pipe"] = lds_pipe(B, per_launch_s)
    # the plain form: its dominant kernel, that kernel's share of the call, and its pipe fraction
    pname, (pcnt, ptot) = max(plain_prof.items(), key=lambda kv: kv[1][1])
    plain["roofline"] = {"kernel": pname, "ms_per_call": ptot / npr,
                         "share_of_call_p50": ptot / npr / plain["p50_ms"],
                         "device_ms_per_call": sum(v[1] for v in plain_prof.values()) / npr}
    if pname == "sample_cand_s3":
        plain["roofline"]["pipe"] = lds_pipe(1, ptot / pcnt / 1000.0)

    line = {"metric": METRIC, "value": ips, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "uint32", "data": "synthetic", "bit_exact": bit_exact,
            "config": {"workload": "N=4096 l=784, x in [0,4], y in [-16,16], 10000 encryptions x 1 key "
                                   "(plain GPU pipeline shape), batched",
                       "n": N, "l": L, "batch": B, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (a batch of ciphertexts is %.1f GB)" % (B * (L + 1) * 3 * N * 4 / 1e9),
                       "randomness": "CPU stream mapping, every stream keyed by a per-encryption seed"},
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "plain": plain, "batched_vs_plain": ips / world / plain["value"],
            "plain_dropin": plain_dropin,
            "batched_vs_plain_dropin": ips / world / plain_dropin["value"] if plain_dropin.get("value") else None,
            "coef0": coef0,
            "batched_vs_plain_forms": {
                "reference_per_call_form": ips / world / plain_dropin["value"] if plain_dropin.get("value") else None,
                "own_per_call_form": ips / world / plain["value"],
                "note": "the 5x target is judged against the reference's plain per-call GPU form (its four entry "
                        "points, one call per encryption, host buffers: plain_dropin); this library's own "
                        "device-resident batch-1 form is bounded near 2.2x by the sigma_3 keystream work "
                        "that every encryption carries"},
            "tuning": {"encrypt_instances_per_group": enc_group, "encrypt_ms_by_group": enc_ms,
                       "coef0_form": c0_form, "coef0_ms_by_form": c0_tune_ms,
                       "coef0_forms": ["per pair", "64x32", "64x64", "32x32", "32x64"],
                       "note": "shapes chosen by the library's tuners (cufe_tune_encrypt, cufe_tune_decrypt_coef0) "
                               "on this workload before timing; every form gives the same bits"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roof,
            "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "clocks": clocks}
    # the other configurations, compact, on the same box (one GPU only): the C2 buffers go first
    if world == 1 and not args.no_extras:
        del ct, dy, res, scratch, r0, pl_ct, pl_dy, pl_out, xd, x_dev, y_dev, sky, mpk, msk
        ctx.close()
        torch.cuda.empty_cache()
        line["c4_ntt"] = ntt_point(4096, 3, 65536, 10, 3)
        mixed = mixed_measure(4096, 5, 3, 24)
        line["c3_batched"] = {k: mixed[k] for k in ("value", "unit", "ms_per_step", "p50_ms", "p99_ms", "bit_exact",
                                                    "setup_s", "graph", "sigma3_samples_per_s", "kernels_ms")}
        line["c3_batched"]["config"] = mixed["config"]
        serve = serve_measure(64, [5000, 10000, 20000, 50000], 0.5, 48, 24, 30,
                              max_tick=args.serve_max_tick, max_queue_s=args.serve_max_queue_ms / 1000.0)
        line["c5_serving"] = {"config": serve["config"], "plain": serve["plain"], "bit_exact": serve["bit_exact"],
                              "results": [{k: r[k] for k in ("rate_rps", "submitted", "completed", "shed",
                                                             "goodput_rps", "bit_exact", "ticks")} |
                                          {"p50_ms": (r["latency"]["all"] or {}).get("p50_ms"),
                                           "p99_ms": (r["latency"]["all"] or {}).get("p99_ms")}
                                          for r in serve["results"]]}
        bit_exact = bit_exact and line["c4_ntt"]["roundtrip_ok"] and mixed["bit_exact"] and serve["bit_exact"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_sample(x, y, seeds2, setup_seeds,
                                                       max(1, min(os.cpu_count() or 1, args.ref_procs)))
        except Exception as e:  # reported, never silently replaced
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1 or args.no_extras:
        ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0 if bit_exact else 1


# ----------------------------------------------------------------------------- kernel sweeps

def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def ntt_sweep(args):
    """Negacyclic NTT and INTT over 65,536 polynomials x n in {1024..8192} x k in {3..6} RNS
    primes (the three params.h primes, then primes 1 mod 16384 below 2^31), residues uniform
    in [0, q_j) from seed 0xC0FE0004.  Each pass reads and writes every residue once: 8n
    bytes per residue polynomial.  All nine kernel variants are timed; the reported figure is
    the one the ring's tuner (cufe_ring_tune) picks.  Every buffer is larger than L2 except n=1024, k=3 at
    fewer polynomials; each timed forward is followed by its inverse and the data must
    come back unchanged."""
    import torch
    import cufe_b200 as cf
    dev = "cuda:0"
    torch.cuda.set_device(0)
    peak = _peaks().get("hbm_gbs", 6650.0)
    g = torch.Generator(device=dev)
    g.manual_seed(0xC0FE0004)
    npoly = args.sweep_polys
    stream = torch.cuda.current_stream()
    clk = Clocks(0, os.path.join(tempfile.gettempdir(), "cufe_clocks_sweep.csv"))
    rows = []
    for n in args.sweep_n:
        for k in args.sweep_k:
            ring = cf.Ring(n, k)
            data = torch.empty((npoly, k, n), dtype=torch.int32, device=dev)
            for j in range(k):
                data[:, j, :] = torch.randint(0, int(ring.primes[j]), (npoly, n), generator=g, device=dev,
                                              dtype=torch.int64).to(torch.int32)
            orig = data.clone()
            nbytes = 8 * n * npoly * k
            per_variant = {}
            ok = True
            for var in args.sweep_variants:
                ring.set_variant(var, var)
                for _ in range(args.warmup):
                    ring.forward(data)
                    ring.inverse(data)
                fwd, inv = [], []
                for _ in range(args.steps):
                    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                    ev[0].record(stream)
                    ring.forward(data)
                    ev[1].record(stream)
                    ring.inverse(data)
                    ev[2].record(stream)
                    torch.cuda.synchronize()
                    fwd.append(ev[0].elapsed_time(ev[1]))
                    inv.append(ev[1].elapsed_time(ev[2]))
                ok = ok and bool(torch.equal(data, orig))
                per_variant[var] = (float(np.median(fwd)), float(np.median(inv)))
            tuned = ring.tune(npoly)
            fv, iv = tuned["variant"]
            if fv not in per_variant or iv not in per_variant:  # a variant left out of the sweep
                fv, iv = (min(per_variant, key=lambda v: per_variant[v][0]),
                          min(per_variant, key=lambda v: per_variant[v][1]))
            f_ms, i_ms = per_variant[fv][0], per_variant[iv][1]
            rows.append({"n": n, "k": k, "bytes_per_pass": nbytes, "fwd_ms": f_ms, "inv_ms": i_ms,
                         "fwd_gbs": nbytes / f_ms / 1e6, "inv_gbs": nbytes / i_ms / 1e6,
                         "fwd_frac": nbytes / f_ms / 1e6 / peak, "inv_frac": nbytes / i_ms / 1e6 / peak,
                         "tuned_variant": [fv, iv],
                         "variants_gbs": {str(v): [nbytes / t[0] / 1e6, nbytes / t[1] / 1e6]
                                          for v, t in per_variant.items()},
                         "roundtrip_ok": ok, "primes": [int(q) for q in ring.primes]})
            del data, orig
            ring.close()
            torch.cuda.empty_cache()
    clocks = clk.stop()
    line = {"workload": "ntt-sweep", "metric": "negacyclic NTT/INTT GB/s (8n bytes per residue polynomial)",
            "unit": "GB/s", "peak": peak, "peak_source": "measured" if "hbm_gbs" in _peaks() else "fallback",
            "polys": npoly, "steps": args.steps, "warmup": args.warmup, "dtype": "uint32", "data": "synthetic",
            "results": rows, "min_frac": min(min(r["fwd_frac"], r["inv_frac"]) for r in rows),
            "all_roundtrips_ok": all(r["roundtrip_ok"] for r in rows), "clocks": clocks}
    print(json.dumps(line), flush=True)
    return 0 if line["all_roundtrips_ok"] else 1


def ntt_point(n, k, npoly, steps, warmup):
    """one point of the kernel sweep with the tuner's variant: forward and inverse negacyclic NTT
    over npoly polynomials of k residues (uniform in [0, q_j), seed 0xC0FE0004), median of
    `steps` event-timed passes, 8n bytes per residue polynomial per pass; the data must come
    back unchanged after every forward + inverse"""
    import torch
    import cufe_b200 as cf
    dev = "cuda:0"
    peak = _peaks().get("hbm_gbs", 6650.0)
    g = torch.Generator(device=dev)
    g.manual_seed(0xC0FE0004)
    ring = cf.Ring(n, k)
    data = torch.empty((npoly, k, n), dtype=torch.int32, device=dev)
    for j in range(k):
        data[:, j, :] = torch.randint(0, int(ring.primes[j]), (npoly, n), generator=g, device=dev,
                                      dtype=torch.int64).to(torch.int32)
    orig = data.clone()
    tuned = ring.tune(npoly)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        ring.forward(data)
        ring.inverse(data)
    fwd, inv = [], []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        ring.forward(data)
        ev[1].record(stream)
        ring.inverse(data)
        ev[2].record(stream)
        torch.cuda.synchronize()
        fwd.append(ev[0].elapsed_time(ev[1]))
        inv.append(ev[1].elapsed_time(ev[2]))
    ok = bool(torch.equal(data, orig))
    nbytes = 8 * n * npoly * k
    f_ms, i_ms = float(np.median(fwd)), float(np.median(inv))
    out = {"n": n, "k": k, "polys": npoly, "bytes_per_pass": nbytes, "fwd_ms": f_ms, "inv_ms": i_ms,
           "fwd_gbs": nbytes / f_ms / 1e6, "inv_gbs": nbytes / i_ms / 1e6,
           "fwd_frac": nbytes / f_ms / 1e6 / peak, "inv_frac": nbytes / i_ms / 1e6 / peak,
           "peak_gbs": peak, "peak_source": "measured" if "hbm_gbs" in _peaks() else "fallback",
           "tuned_variant": list(tuned["variant"]), "roundtrip_ok": ok}
    del data, orig
    ring.close()
    torch.cuda.empty_cache()
    return out


def sampler_sweep(args):
    """2^30 discrete Gaussian samples per sigma in both mappings at n = 4096: samples/s over
    the sampler launches (CUDA events) and Pearson chi-square on 1000 equiprobable bins of
    the ideal D_{Z,sigma}.  The reference's sigma_2 and sigma_3 samplers are not
    D_{Z,sigma} (their Bernoulli input conversion is exact only below 2^52), and the kernels
    reproduce them bit for bit, so only sigma_1 is expected to pass against the ideal."""
    import torch
    import cufe_b200 as cf
    from cufe_b200.stats import ChiSquare, sigma_of, signed_samples
    torch.cuda.set_device(0)
    n = 4096
    ctx = cf.Context(n, 8, device=0)
    rng = np.random.default_rng(0xC0FE0004)
    total = args.sweep_samples
    stream = torch.cuda.current_stream()
    clk = Clocks(0, os.path.join(tempfile.gettempdir(), "cufe_clocks_sampler.csv"))
    rows = []
    for mapping in ("cpu", "gpu"):
        for sig in range(3):
            acc = ChiSquare(sigma_of(sig), 1000)
            ms, done = 0.0, 0
            if mapping == "cpu":
                ns, calls = 64, 512
                out = torch.empty((ns, calls, 3, n), dtype=torch.int32, device="cuda:0")
            else:
                npolys = 32768
                out = torch.empty((npolys, 3, n), dtype=torch.int32, device="cuda:0")
            per = out.numel() // 3
            warm = True
            while done < total:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if mapping == "cpu":
                    ctx.sample_cpu_map(sig, rng.integers(0, 256, (ns, 32), dtype=np.uint8), calls, out=out)
                else:
                    ctx.sample_gpu_map(sig, rng.integers(0, 256, 32, dtype=np.uint8), 0, npolys, out=out)
                e1.record(stream)
                torch.cuda.synchronize()
                if warm:  # first chunk: warm-up, not counted
                    warm = False
                    continue
                ms += e0.elapsed_time(e1)
                acc.add(signed_samples(out))
                done += per
            res = acc.result()
            rows.append({"mapping": mapping, "sigma_index": sig, "sigma": sigma_of(sig), "samples": done,
                         "samples_per_s": done / (ms / 1000.0), "gb_per_s_out": 12 * done / (ms / 1000.0) / 1e9,
                         "chi2_ideal": {k: res[k] for k in ("chi2", "df", "p_value", "bins", "worst_bins")}})
            del out
            torch.cuda.empty_cache()
    clocks = clk.stop()
    ctx.close()
    line = {"workload": "sampler-sweep", "metric": "discrete Gaussian samples/s at n=4096 (12 B of residues each)",
            "unit": "samples/s", "dtype": "int64 samples, uint32 residues", "data": "synthetic",
            "results": rows, "clocks": clocks,
            "note": "sigma_2/sigma_3 deviate from the ideal in the reference itself; tests check them "
                    "against the reference's own distribution (two-sample chi-square)"}
    print(json.dumps(line), flush=True)
    return 0


def splitmix64(x):
    """one SplitMix64 output for state x (Steele, Lea, Flood 2014)"""
    m = (1 << 64) - 1
    z = (x + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def batched_mixed(args):
    """the heterogeneous batch as its own workload line (see mixed_measure)"""
    import torch
    torch.cuda.set_device(0)
    line = mixed_measure(args.instances, args.steps, args.warmup, args.chunk_gb)
    print(json.dumps(line), flush=True)
    return 0 if line["bit_exact"] else 1


def mixed_measure(count, steps, warmup, chunk_gb, tune_gb=(12, 24, 36)):
    """Heterogeneous batch: `count` independent IPFE instances, l = round(exp(U[ln 32, ln 1024])),
    N in {2048, 4096} 50/50, x in [0, 4], y in [-16, 16]; instance i's data from
    SplitMix64(0xC0FE0003 + i).  Keys are generated once (setup timed separately) and stay
    resident; a step is one replay of the batch's CUDA graph (encrypt + keygen + decrypt +
    decode of every instance) with fresh encryption seeds copied in from pinned host memory.
    Every inner product of the timed steps is checked against the plaintext dot product.
    Launch gaps: one more step runs eagerly with CUDA events around every kernel group;
    replay time / summed kernel time is the graph's cost over its kernels."""
    import torch
    import cufe_b200 as cf
    ns, ls, xs, ys, seeds = [], [], [], [], []
    for i in range(count):
        r = np.random.default_rng(splitmix64(0xC0FE0003 + i))
        ls.append(int(round(float(np.exp(r.uniform(np.log(32), np.log(1024)))))))
        ns.append(2048 if r.random() < 0.5 else 4096)
        xs.append(r.integers(0, 5, ls[-1]))
        ys.append(r.integers(-16, 17, ls[-1]))
        seeds.append(r.integers(0, 256, (3, 32), dtype=np.uint8))
    seeds = np.stack(seeds)
    t0 = time.perf_counter()
    B = cf.Batch(ns, ls, max_chunk_bytes=chunk_gb << 30)
    B.setup(seeds[:, 0], seeds[:, 1], seeds[:, 2])
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    x = cf.to_dev(B.pack(xs).astype(np.uint32))
    y = cf.to_dev(B.pack(ys).astype(np.int32))
    rng = np.random.default_rng(0xC0FE0003)
    total = warmup + steps + 1
    host_seeds = torch.from_numpy(rng.integers(0, 256, (total, 2, count, 32), dtype=np.uint8)).pin_memory()
    s2 = torch.empty((count, 32), dtype=torch.uint8, device="cuda:0")
    s3 = torch.empty_like(s2)
    out = B.bind(x, y, s2, s3)
    res = torch.empty((steps + 1, count), dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream()

    def seeds_in(k):
        s2.copy_(host_seeds[k, 0], non_blocking=True)
        s3.copy_(host_seeds[k, 1], non_blocking=True)

    seeds_in(0)
    budgets = [b << 30 for b in tune_gb] if tune_gb else []
    chunk_choice = B.tune(budgets) if budgets else (chunk_gb << 30, [])
    for k in range(warmup):
        seeds_in(k)
        B.replay()
    torch.cuda.synchronize()
    B.status()
    clk = Clocks(0, os.path.join(tempfile.gettempdir(), "cufe_clocks_mixed.csv"))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        seeds_in(warmup + k)
        B.replay()
        res[k].copy_(out)
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    B.status()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    ms = ev[0].elapsed_time(ev[steps])
    # one eager step with kernel timing: the replay's launch gaps against its kernel time
    seeds_in(warmup + steps)
    torch.cuda.synchronize()
    B.profile(True)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    B.run()
    g1.record(stream)
    res[steps].copy_(out)
    torch.cuda.synchronize()
    kernel_ms, kernels = B.profile_read()
    groups = B.profile_groups()
    B.profile(False)
    eager_ms = g0.elapsed_time(g1)
    p = np.array([64 * l + 1 for l in ls], np.int64)
    exp = np.array([int(a @ b) for a, b in zip(xs, ys)], np.int64) % p
    got = cf.u32(res).astype(np.int64) % p[None, :]
    ok = bool((got == exp[None, :]).all())
    samples = sum(l * n for l, n in zip(ls, ns))
    replay_ms = float(np.median(step_ms))
    line = {"workload": "batched-mixed", "metric": "IPFE inner products/sec, heterogeneous batch (bit-exact)",
            "value": steps * count / (ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": steps,
            "warmup": warmup, "ms_per_step": ms / steps, "p50_ms": float(np.percentile(step_ms, 50)),
            "p99_ms": float(np.percentile(step_ms, 99)), "higher_is_better": True, "dtype": "uint32",
            "data": "synthetic", "bit_exact": ok, "setup_s": setup_s,
            "graph": {"kernels": B.graph_kernels(), "replay_ms": replay_ms,
                      "eager_kernel_ms": kernel_ms, "eager_kernels": kernels, "eager_step_ms": eager_ms,
                      "replay_over_kernel_time": replay_ms / kernel_ms if kernel_ms else None,
                      "note": "kernel time from CUDA events around every kernel group of one eager step"},
            "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in sorted(groups.items(), key=lambda kv: -kv[1][1])},
            "config": {"workload": "%d instances, l log-uniform [32, 1024], N 2048/4096 50/50, one CUDA graph "
                                   "replay per step" % count,
                       "instances": count, "mean_l": float(np.mean(ls)), "n4096_share": float(np.mean(np.array(ns) == 4096)),
                       "chunks": B.chunks, "key_gb": B.key_bytes / 1e9, "scratch_gb": B.scratch_bytes / 1e9,
                       "chunk_budget_gb": chunk_choice[0] / (1 << 30),
                       "chunk_tuning_ms": dict(zip([str(b) for b in tune_gb], chunk_choice[1])) if budgets else None,
                       "sigma3_samples_per_step": samples},
            "sigma3_samples_per_s": samples / (ms / steps / 1000.0), "clocks": clocks}
    B.close()
    return line


def serving(args):
    """the serving loop as its own workload line (see serve_measure)"""
    import torch
    torch.cuda.set_device(0)
    line = serve_measure(args.tenants, args.rates, args.duration, args.arena_gb, args.tick_gb,
                         args.plain_requests, args.max_tick, args.max_queue_ms / 1000.0)
    print(json.dumps(line), flush=True)
    return 0 if line["bit_exact"] else 1


def serve_measure(T, rates, duration, arena_gb, tick_gb, plain_requests, max_tick=0, max_queue_s=0.0):
    """Serving loop: open-loop Poisson arrivals at each rate for `duration` seconds, request mix
    encrypt:keygen:decrypt = 4:1:4, T tenants with l log-uniform in [64, 1024] and N in
    {2048, 4096} (keys resident), seeded from SplitMix64(0xC0FE0005 + i).  Decryptions read a
    resident pool of ciphertexts and function keys per tenant (their inner products are
    checked); new ciphertexts and keys are released as they complete.  Latency = completion
    seen by the server's poll minus the scheduled arrival time, over completed requests.
    With overload limits (max_tick requests per tick, max_queue_s of queueing) requests that
    waited too long are shed; goodput counts completed requests only.  The plain form serves
    a sample of the same requests one per tick, each to completion, on the same kernels."""
    import cufe_b200 as cf
    ns, ls = [], []
    for i in range(T):
        r = np.random.default_rng(splitmix64(0xC0FE0005 + i))
        ls.append(int(round(float(np.exp(r.uniform(np.log(64), np.log(1024)))))))
        ns.append(2048 if r.random() < 0.5 else 4096)
    rng = np.random.default_rng(0xC0FE0005)
    S = cf.Server(ns, ls, arena_bytes=arena_gb << 30, tick_bytes=tick_gb << 30)
    S.setup(rng.integers(0, 256, (T, 32), dtype=np.uint8), None, rng.integers(0, 256, (T, 32), dtype=np.uint8))
    # resident pool: 2 ciphertexts and 2 function keys per tenant
    pool = []
    for t in range(T):
        xs = [rng.integers(0, 5, ls[t]).astype(np.uint32) for _ in range(2)]
        ys = [rng.integers(-16, 17, ls[t]).astype(np.int32) for _ in range(2)]
        cts = [S.encrypt(t, x, rng.integers(0, 256, 32, dtype=np.uint8), rng.integers(0, 256, 32, dtype=np.uint8))
               for x in xs]
        sks = [S.keygen(t, y) for y in ys]
        pool.append((xs, ys, cts, sks))
    S.drain()
    S.limits(max_tick, max_queue_s)
    kinds = np.array([0] * 4 + [1] + [2] * 4)

    def make_requests(k, rate):
        gaps = rng.exponential(1.0 / rate, k)
        when = np.cumsum(gaps)
        reqs = []
        for i in range(k):
            kind = int(kinds[rng.integers(0, 9)])
            t = int(rng.integers(0, T))
            if kind == 0:
                reqs.append((when[i], 0, t, rng.integers(0, 5, ls[t]).astype(np.uint32),
                             rng.integers(0, 256, 32, dtype=np.uint8), rng.integers(0, 256, 32, dtype=np.uint8)))
            elif kind == 1:
                reqs.append((when[i], 1, t, rng.integers(-16, 17, ls[t]).astype(np.int32)))
            else:
                reqs.append((when[i], 2, t, int(rng.integers(0, 2)), int(rng.integers(0, 2))))
        return reqs

    def submit(req, t_arr):
        if req[1] == 0:
            return S.encrypt(req[2], req[3], req[4], req[5], t_arr)
        if req[1] == 1:
            return S.keygen(req[2], req[3], t_arr)
        xs, ys, cts, sks = pool[req[2]]
        return S.decrypt(cts[req[3]], sks[req[4]], t_arr)

    def check(req, rid):
        """(finished state is valid and a decrypt's value is right, completed, latency ms)"""
        st, v, ta, td = S.result(rid)
        if st == S.SHED:
            return True, False, None
        ok = st in (S.DONE, S.RELEASED)
        if req[1] == 2:
            xs, ys, _, _ = pool[req[2]]
            p = 64 * ls[req[2]] + 1
            ok = ok and v % p == int(xs[req[3]].astype(np.int64) @ ys[req[4]].astype(np.int64)) % p
        return ok, True, 1000.0 * (td - ta)

    def release_finished(owned):
        while owned:
            st = S.result(owned[0])[0]
            if st not in (S.DONE, S.SHED):
                return
            rid = owned.pop(0)
            if st == S.DONE:
                S.release(rid)

    results = []
    for rate in rates:
        reqs = make_requests(max(1, int(rate * duration)), rate)
        t0 = S.now() + 0.01
        ids, owned = [], []
        t_pos = 0
        t_stat0 = S.stats()
        while t_pos < len(reqs):
            now = S.now()
            while t_pos < len(reqs) and t0 + reqs[t_pos][0] <= now:
                rid = submit(reqs[t_pos], t0 + reqs[t_pos][0])
                ids.append(rid)
                if reqs[t_pos][1] != 2:
                    owned.append(rid)
                t_pos += 1
            S.poll()
            release_finished(owned)  # bound the arenas
        while True:
            q, fl = S.pending()
            release_finished(owned)
            if q == 0 and fl == 0:
                break
            S.poll(wait=fl > 0)
        lat = {0: [], 1: [], 2: []}
        ok, completed, t_end = True, 0, t0
        for req, rid in zip(reqs, ids):
            good, done, ms = check(req, rid)
            ok = ok and good
            if done:
                completed += 1
                lat[req[1]].append(ms)
                t_end = max(t_end, S.result(rid)[3])
        for rid in owned:
            if S.result(rid)[0] == S.DONE:
                S.release(rid)
        st = S.stats()
        allv = lat[0] + lat[1] + lat[2]
        pct = lambda v: {"p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99)),  # noqa: E731
                         "n": len(v)} if v else None
        span = max(t_end - t0, 1e-9)
        results.append({"rate_rps": rate, "submitted": len(reqs), "completed": completed,
                        "shed": st["shed"] - t_stat0["shed"], "bit_exact": ok,
                        "goodput_rps": completed / span, "span_s": span,
                        "latency": {"all": pct(allv), "encrypt": pct(lat[0]), "keygen": pct(lat[1]),
                                    "decrypt": pct(lat[2])},
                        "ticks": st["ticks"] - t_stat0["ticks"],
                        "requests_per_tick": completed / max(1, st["ticks"] - t_stat0["ticks"])})
    S.limits(0, 0.0)
    # plain per-call form: one request per tick, run to completion, same kernels
    sample = make_requests(plain_requests, 1000.0)
    plat = []
    for req in sample:
        t_a = S.now()
        rid = submit(req, t_a)
        S.drain()
        good, _, ms = check(req, rid)
        plat.append(ms)
        if req[1] != 2:
            S.release(rid)
    plain = {"throughput_rps": 1000.0 * len(plat) / sum(plat), "p50_ms": float(np.percentile(plat, 50)),
             "p99_ms": float(np.percentile(plat, 99)), "requests": len(plat),
             "form": "one request per tick, submitted and run to completion before the next"}
    line = {"workload": "serving", "metric": "requests/s and p50/p99 latency, encrypt:keygen:decrypt = 4:1:4",
            "unit": "req/s", "n_gpus": 1, "data": "synthetic", "dtype": "uint32",
            "config": {"tenants": T, "mean_l": float(np.mean(ls)), "n4096_share": float(np.mean(np.array(ns) == 4096)),
                       "duration_s": duration, "arena_gb": arena_gb, "tick_gb": tick_gb,
                       "max_tick_requests": max_tick, "max_queue_ms": 1000.0 * max_queue_s},
            "results": results, "plain": plain,
            "bit_exact": all(r["bit_exact"] for r in results)}
    S.close()
    return line


def _svm_ref_init(path):
    global _SREF, _SDATA
    from oracle.ffi import Reference
    _SREF = Reference("n2048_l124")
    d = np.load(path)
    _SDATA = {k: d[k] for k in d.files}


def _svm_ref_one(t):
    """svm_predict3 for one test vector on the reference CPU build: encrypt, then for every
    support vector keygen + decrypt + GMP decode (y split into y+ - y-, as the reference
    reduces y as uint32), then the vote"""
    d = _SDATA
    ct = _SREF.encrypt(d["x"][t], d["mpk"], d["s2"][t])
    p = 64 * 124 + 1
    kv = []
    for i in range(d["svp"].shape[0]):
        _, dp = _SREF.decrypt(ct, d["svp"][i], _SREF.keygen(d["svp"][i], d["msk"]))
        _, dm = _SREF.decrypt(ct, d["svm"][i], _SREF.keygen(d["svm"][i], d["msk"]))
        v = (int(dp[0]) - int(dm[0])) % p
        kv.append(v - p if v > p // 2 else v)
    s = float(np.dot(d["coef"][0][:250], kv[:250]) + np.dot(d["coef"][0][250:], kv[250:])) - float(d["rho"][0])
    return 1 if s > 0 else -1


def svm_workload(args):
    """Plain IPFE-SVM prediction (the svm_predict3 / svm_predict5 shape): N = 2048, the params.h
    primes, l = 124 (123 features at 1-based indices), 1,000 test vectors x in {0,1}^123 with 14
    ones at uniform positions, a linear two-class model of 500 support vectors with integer
    weights in [-16, 16] (250 per class, sv_coef uniform, rho uniform), data from
    SplitMix64(0xC0FE0001).  Keys: one master key; the support vectors' function keys are
    derived once (timed separately).  A step encrypts all 1,000 test vectors and predicts them
    (coefficient-0 decryption of every (test vector, support vector) pair + the vote).  Every
    inner product and label of the timed steps is checked against the plaintext model."""
    import torch
    import cufe_b200 as cf
    n, l, ntest, nsv = 2048, 124, 1000, 500
    rng = np.random.default_rng(splitmix64(0xC0FE0001))
    x = np.zeros((ntest, l), np.uint32)
    for t in range(ntest):
        x[t, 1 + rng.choice(123, 14, replace=False)] = 1
    sv = np.zeros((nsv, l), np.int32)
    sv[:, 1:] = rng.integers(-16, 17, (nsv, 123))
    coef = np.concatenate([rng.uniform(0, 1, 250), -rng.uniform(0, 1, 250)])[None, :]
    rho = rng.uniform(-1, 1, 1)
    label = np.array([1, -1], np.int32)
    seeds_setup = rng.integers(0, 256, (2, 32), dtype=np.uint8)
    s2 = rng.integers(0, 256, (args.warmup + args.steps, ntest, 32), dtype=np.uint8)
    torch.cuda.set_device(0)
    c = cf.Context(n, l)
    mpk, msk = c.setup(seeds_setup[0], None, seeds_setup[1])
    t0 = time.perf_counter()
    m = cf.SvmModel(c, sv, [250, 250], coef, rho, label, msk, signed=True)
    keys_s = time.perf_counter() - t0
    xd = cf.to_dev(x)
    ct = c.ct_buf(ntest)
    kv = torch.empty((ntest, nsv), dtype=torch.int32, device="cuda:0")
    labels = torch.empty((args.steps, ntest), dtype=torch.int32, device="cuda:0")
    kvs = []
    stream = torch.cuda.current_stream()

    def step(k, out, kvo):
        c.encrypt(xd, mpk, s2[k], None, ct=ct)
        m.predict(ct, labels=out, kvalue=kvo)

    c.encrypt(xd, mpk, s2[0], None, ct=ct)
    svm_form, svm_form_ms = m.tune(ct)  # the coefficient-0 decrypt form for 1,000 x 500 pairs
    for k in range(args.warmup):
        step(k, labels[0], kv)
    c.sync()
    clk = Clocks(0, os.path.join(tempfile.gettempdir(), "cufe_clocks_svm.csv"))
    c.profile_reset()
    c.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(args.warmup + k, labels[k], kv)
        if k == args.steps - 1:
            kvs.append(kv.clone())
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    c.profile(False)
    prof = c.profile_read()
    svm_launches = c.profile_launches()
    ms = e0.elapsed_time(e1)
    p = 64 * l + 1
    ip = x.astype(np.int64) @ sv.astype(np.int64).T
    kvh = cf.u32(kvs[0]).astype(np.int64)
    kvh = np.where(kvh > p // 2, kvh - p, kvh)
    dv = (ip[:, :250].astype(np.float64) @ coef[0][:250] + ip[:, 250:].astype(np.float64) @ coef[0][250:]) - rho[0]
    want = np.where(dv > 0, 1, -1)
    ok = bool((kvh == ip).all()) and bool((labels.cpu().numpy() == want[None, :]).all())
    preds = args.steps * ntest / (ms / 1000.0)
    line = {"workload": "svm", "metric": "encrypted SVM predictions/s (N=2048, l=124, 500 SVs; bit-exact)",
            "value": preds, "unit": "predictions/s", "ip_per_s": preds * nsv, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "uint32",
            "data": "synthetic", "bit_exact": ok, "sv_keys_s": keys_s,
            "tuning": {"coef0_form": svm_form, "coef0_ms_by_form": svm_form_ms,
                       "coef0_forms": ["per pair", "64x32", "64x64", "32x32", "32x64"]},
            "config": {"workload": "1,000 test vectors (a1a-shaped) x 500 support vectors, encrypt + predict per step",
                       "n": n, "l": l, "test_vectors": ntest, "support_vectors": nsv},
            "gpu_launches": svm_launches, "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "clocks": clocks}
    if not args.no_cpu_baseline:
        import multiprocessing as mp
        from oracle.ffi import Reference
        R = Reference("n2048_l124")
        rmpk, rmsk = R.setup(seeds_setup[0], seeds_setup[1])
        tmp = tempfile.NamedTemporaryFile(suffix=".npz", delete=False)
        np.savez(tmp.name, x=x, mpk=rmpk, msk=rmsk, s2=s2[0], svp=np.where(sv > 0, sv, 0).astype(np.uint32),
                 svm=np.where(sv < 0, -sv, 0).astype(np.uint32), coef=coef, rho=rho)
        nproc = max(1, min(os.cpu_count() or 1, args.ref_procs))
        pool = mp.get_context("spawn").Pool(nproc, initializer=_svm_ref_init, initargs=(tmp.name,))
        try:
            t0 = time.perf_counter()
            res = pool.map(_svm_ref_one, list(range(nproc)))
            dt = time.perf_counter() - t0
        finally:
            pool.terminate()
            os.unlink(tmp.name)
        line["cpu_baseline"] = {"value": nproc / dt, "unit": "predictions/s", "cores": nproc, "kind": "reference",
                                "sample": "%d test vectors, one per process: encrypt + 500 x (2 keygens + 2 decrypts "
                                          "+ GMP decode) + vote (svm_predict3 structure)" % nproc,
                                "labels_match": bool((np.array(res) == want[:nproc]).all())}
    print(json.dumps(line), flush=True)
    m.close()
    c.close()
    return 0 if ok else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=200)
    ap.add_argument("--impl", default="cufe", choices=["cufe", "reference"])
    ap.add_argument("--plain-calls", type=int, default=30)
    ap.add_argument("--dropin-calls", type=int, default=20)
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="pipeline",
                    choices=["pipeline", "ntt-sweep", "sampler-sweep", "batched-mixed", "serving", "svm"])
    ap.add_argument("--tenants", type=int, default=64)
    ap.add_argument("--rates", type=lambda v: [float(t) for t in v.split(",")], default=[5000, 10000, 20000, 50000])
    ap.add_argument("--duration", type=float, default=1.0)
    ap.add_argument("--arena-gb", type=int, default=48)
    ap.add_argument("--tick-gb", type=int, default=24)
    ap.add_argument("--plain-requests", type=int, default=100)
    ap.add_argument("--max-tick", type=int, default=0, help="serving: requests per tick (0: memory only)")
    ap.add_argument("--max-queue-ms", type=float, default=0.0, help="serving: shed requests queued longer")
    ap.add_argument("--no-extras", action="store_true", help="pipeline: skip the C3/C4/C5 sub-measurements")
    ap.add_argument("--serve-max-tick", type=int, default=512, help="pipeline's serving sub-line: per-tick cap")
    ap.add_argument("--serve-max-queue-ms", type=float, default=50.0, help="pipeline's serving sub-line: deadline")
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--chunk-gb", type=int, default=24)
    ap.add_argument("--sweep-polys", type=int, default=65536)
    ap.add_argument("--sweep-samples", type=int, default=2 ** 30)
    ints = lambda v: [int(t) for t in v.split(",")]  # noqa: E731
    ap.add_argument("--sweep-n", type=ints, default=[1024, 2048, 4096, 8192])
    ap.add_argument("--sweep-k", type=ints, default=[3, 4, 5, 6])
    ap.add_argument("--sweep-variants", type=ints, default=list(range(1, 10)))
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "ntt-sweep":
        return ntt_sweep(args)
    if args.workload == "sampler-sweep":
        return sampler_sweep(args)
    if args.workload == "batched-mixed":
        return batched_mixed(args)
    if args.workload == "serving":
        return serving(args)
    if args.workload == "svm":
        return svm_workload(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
