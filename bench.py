#!/usr/bin/env python
"""E8Q IVF search on B200 -- benchmark (one JSON line on rank 0).

Workload (N=1 headline): 1M x 960-d float32 base drawn on the GPU from a
seeded 1,024-component Gaussian mixture (centres N(0, diag(lambda)), members
centre + 0.4 N(0, diag(lambda)), lambda_i ~ i^-0.5 normalised to mean 1; the
sqrt(lambda) scaling applies to both draws), cluster_ids = generating
component, centroids = per-list means; 10,240 queries from the same mixture;
E8Q nbits=6 (the lowest rate whose recall@10 clears 0.95 on this mixture),
k=10, nprobe=64; one step = one batch of 4,096 queries through the search
path (default --path precision: int8 tensor-core candidates + exact
rescoring; --path batched / plain measure the other modes). Synthetic data
stands in for the public corpora (no network).

  value  : QPS with queries already in HBM (E8qIndex.search_ptr), CUDA events
           on the launching stream, max over ranks; --gpus N runs N replicas
           (the index fits one GPU; no data-path collective), scaling "weak".
  e2e    : the same QPS through E8qIndex.search(numpy) with pinned host query
           buffers: H2D of the queries and D2H of ids+dists inside the timing
           (events; host_wall_qps is the same loop by the host clock).
  roofline: the dominant scan kernel's algorithmic bytes per launch over its
           CUDA-event time against the measured HBM copy bandwidth -- for the
           precision scan: int8 proxy row + g1/h3 per vector of each work item
           plus 2 bytes of fp16 proxy distance written per (query, vector) pair;
           beside it the int8 tensor ops against an int8 MMA rate measured in
           the run with the library's tcgen05 probe.
  plain_gpu_qps: the plain one-query-per-launch GPU scan on the same index.
  pruned_gpu_qps: the reference's search semantics on the GPU (mode "pruned",
                  E8qIndex.search's default) on one batch of queries.
  serving: open-loop Poisson load through e8qlib.Server (U{1..64} queries per
           request) at fractions of `value`: achieved QPS, p50/p99/max ms;
           the loads with the headline k and nprobe, then one of uneven
           requests (k in {10, 100}, nprobe in {16, 32, 64} drawn per request).
  --sweep: the nbits x nprobe grid, query-batch sweeps and the other E8Q
           configurations instead of the bench line (see run_sweep).
  cpu_baseline: the reference's own CPU search (compiled from its sources into
           oracle/_ref), all host cores, a bounded sample of the same workload.

--impl reference times that reference CPU search as the measured arm.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "e8q-artifact_b200"))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--path", choices=["plain", "batched", "precision"], default="precision")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=960)
    ap.add_argument("--nlist", type=int, default=1024)
    ap.add_argument("--nbits", type=int, default=6)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--nprobe", type=int, default=64)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--pool", type=int, default=10240)
    ap.add_argument("--gt", type=int, default=1000, help="queries with FP64 ground truth")
    ap.add_argument("--plain-batch", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the open-loop serving leg")
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--serve-loads", default="0.3,0.6", help="offered load as fractions of the batch QPS")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-me8q", action="store_true", help="skip the ME8Q leg")
    ap.add_argument("--me8q-n", type=int, default=10_000_000)
    ap.add_argument("--me8q-dim", type=int, default=768)
    ap.add_argument("--me8q-nlist", type=int, default=4096)
    ap.add_argument("--me8q-avg-bits", default="4,6", help="comma-separated avg_bits values")
    ap.add_argument("--me8q-nprobes", default="32,64,128,256,512")
    ap.add_argument("--me8q-lloyd", type=int, default=3, help="Lloyd steps refining the ME8Q lists")
    ap.add_argument("--spectrum", type=float, default=0.5, help="per-dimension variance lambda_i ~ i^-spectrum")
    ap.add_argument("--sigma", type=float, default=0.4, help="within-component standard deviation")
    ap.add_argument("--sweep", action="store_true",
                    help="instead of the bench line: nbits x nprobe grid, batch sizes and the 100k x 128 "
                         "config, one JSON line")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def int8_peak(device):
    """Dense int8 tensor-core rate (TOPS, 2 ops per multiply-add) of this GPU,
    measured with the library's tcgen05 kind::i8 probe: one CTA per SM, each
    issuing back-to-back 128x256x256 MMAs from shared memory."""
    import e8qlib
    import torch

    sms = torch.cuda.get_device_properties(device).multi_processor_count
    rng = np.random.default_rng(0)
    A = rng.integers(-8, 8, (128, 256), dtype=np.int8)
    B = rng.integers(-8, 8, (256, 256), dtype=np.int8)
    reps = 4000
    e8qlib.tc_i8_gemm(A, B, reps=10, grid=sms, device=device)
    best = 0.0
    for _ in range(3):
        _, ms = e8qlib.tc_i8_gemm(A, B, reps=reps, grid=sms, device=device)
        best = max(best, 2.0 * 128 * 256 * 256 * reps * sms / (ms / 1000.0) / 1e12)
    return best


def workload_name(a):
    return (f"E8Q IVF search, {a.n // 1000}k x {a.dim}-d Gaussian mixture ({a.nlist} lists, "
            f"sigma {a.sigma}, lambda_i ~ i^-{a.spectrum}), nbits={a.nbits}, k={a.k}, nprobe={a.nprobe}, "
            f"query batch {a.batch}")


def gen_data(a, device, rank):
    """The mixture on `device` (torch), seeded; queries differ per rank."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(1000 + a.seed)
    lam = torch.arange(1, a.dim + 1, device=device, dtype=torch.float64) ** -getattr(a, "spectrum", 0.5)
    lam = lam / lam.mean()
    s = lam.sqrt().float()
    cen = torch.randn(a.nlist, a.dim, generator=g, device=device) * s
    lab = torch.randint(0, a.nlist, (a.n,), generator=g, device=device)
    x = torch.empty(a.n, a.dim, device=device)
    step = 1 << 18
    for i in range(0, a.n, step):
        j = min(a.n, i + step)
        x[i:j] = cen[lab[i:j]] + getattr(a, "sigma", 0.4) * torch.randn(j - i, a.dim, generator=g, device=device) * s
    cm = torch.zeros(a.nlist, a.dim, device=device, dtype=torch.float64)
    cm.index_add_(0, lab, x.double())
    cnt = torch.bincount(lab, minlength=a.nlist).clamp_min(1).double()
    cm = (cm / cnt[:, None]).float()
    gq = torch.Generator(device=device)
    gq.manual_seed(2000 + a.seed + 7919 * rank)
    lq = torch.randint(0, a.nlist, (a.pool,), generator=gq, device=device)
    q = cen[lq] + getattr(a, "sigma", 0.4) * torch.randn(a.pool, a.dim, generator=gq, device=device) * s
    return x.contiguous(), cm.contiguous(), lab.to(torch.int32).contiguous(), q.contiguous()


def ground_truth(x, q, k):
    """FP64 brute-force top-k over the raw vectors (base in chunks of 1M rows)."""
    import torch

    best_d, best_i = None, None
    for c0 in range(0, x.shape[0], 1 << 20):
        xd = x[c0:c0 + (1 << 20)].double()
        xn = (xd * xd).sum(1)
        dd, ii = [], []
        for i in range(0, q.shape[0], 256):
            qd = q[i:i + 256].double()
            d = (qd * qd).sum(1, keepdim=True) + xn[None, :] - 2.0 * qd @ xd.T
            t = torch.topk(d, min(k, d.shape[1]), dim=1, largest=False)
            dd.append(t.values)
            ii.append(t.indices + c0)
        dd, ii = torch.cat(dd), torch.cat(ii)
        if best_d is None:
            best_d, best_i = dd, ii
        else:
            cd, ci = torch.cat([best_d, dd], 1), torch.cat([best_i, ii], 1)
            t = torch.topk(cd, k, dim=1, largest=False)
            best_d, best_i = t.values, torch.gather(ci, 1, t.indices)
        del xd
    return best_i.cpu().numpy()


def recall_at(ids, gt, k=10):
    hit = 0
    for r, g in zip(ids[:, :k], gt[:, :k]):
        hit += len(set(r.tolist()) & set(g.tolist()))
    return hit / (gt.shape[0] * k)


def host_cpu():
    """Threads the CPU baseline uses and what they are: one per physical core
    available to this process (logical CPUs in the affinity mask divided by
    the hardware threads per core), the logical count and the CPU model."""
    logical = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil

        per_core = max(1, (psutil.cpu_count(logical=True) or 1) // max(1, psutil.cpu_count(logical=False) or 1))
    except Exception:
        per_core = 1
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cores": max(1, logical // per_core), "logical_cpus": logical, "threads_per_core": per_core,
            "cpu_model": model}


def time_rounds(fn, nq, warmup=3, min_rounds=9, min_s=0.4, max_s=30.0):
    """QPS of fn() (nq queries per call) with the reference protocol's timing
    (experiments/protocol.py:559-597): `warmup` untimed calls, then rounds
    until at least min_rounds rounds and min_s seconds; median QPS with p25 and
    p75. max_s bounds the host time of slow arms (at least 3 rounds)."""
    for _ in range(warmup):
        fn()
    qps = []
    t_start = time.perf_counter()
    while len(qps) < min_rounds or time.perf_counter() - t_start < min_s:
        t0 = time.perf_counter()
        fn()
        qps.append(nq / (time.perf_counter() - t0))
        if time.perf_counter() - t_start > max_s and len(qps) >= 3:
            break
    qps.sort()
    return {"qps": statistics.median(qps), "p25": float(np.percentile(qps, 25)),
            "p75": float(np.percentile(qps, 75)), "rounds": len(qps)}


def relerr(x, q, ids, dists, k):
    """SAQ relative distance error |D_hat - Delta| / Delta over the returned
    top-k (experiments/protocol.py:525-556, p99 as in :941-966): D_hat is the
    distance the search returned for an id, Delta the exact squared L2 from the
    raw vectors in FP64. Returns (mean, p99, max)."""
    import torch

    idt = torch.from_numpy(ids[:, :k].astype(np.int64)).to(x.device)
    dt = torch.from_numpy(np.ascontiguousarray(dists[:, :k])).to(x.device).double()
    ok = (idt >= 0) & (idt < x.shape[0]) & torch.isfinite(dt)
    errs = []
    for i in range(0, idt.shape[0], 128):
        ii = idt[i:i + 128].clamp(0, x.shape[0] - 1)
        delta = ((q[i:i + 128, None, :].double() - x[ii].double()) ** 2).sum(-1)
        m = ok[i:i + 128] & (delta > 1e-12)
        errs.append(((dt[i:i + 128] - delta).abs() / delta)[m])
    e = torch.cat(errs).cpu().numpy()
    if e.size == 0:
        return -1.0, -1.0, -1.0
    return float(e.mean()), float(np.percentile(e, 99)), float(e.max())


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.p = None
        import tempfile

        fd, self.path = tempfile.mkstemp(prefix=f"e8q_clocks_{dev}_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap,utilization.gpu",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            time.sleep(0.15)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [t.strip() for t in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:7], float(parts[7])))
            except ValueError:
                continue
        os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        busy = [r for r in rows if r[3] > 0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in busy for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(busy)}


def plain_roofline(prof, a, peak, pk_kind):
    """The plain scan kernel (one query per launch) against HBM: algorithmic
    bytes per launch = (nbits * Dpad / 8 + 8) per candidate (codes, g1, h3);
    its CUDA-event time per launch; beside it the whole per-query chain
    (routing launch + scan launch) with the route sweep's nlist * Dpad * 4
    bytes added."""
    n = max(1, prof["scan_launches"])
    t = prof["scan_ms"] / n / 1000.0
    b = prof["algo_bytes"] / n
    pd = (a.dim + 63) // 64 * 64
    rb = a.nlist * pd * 4 + a.nlist * 4
    tr = prof["prep_ms"] / n / 1000.0
    ach = b / t / 1e9 if t > 0 else 0.0
    chain = (b + rb) / (t + tr) / 1e9 if t + tr > 0 else 0.0
    return {"kernel": "scan_plain_kernel", "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
            "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": pk_kind,
            "algo_bytes_per_launch": int(b), "launch_us": round(t * 1e6, 2),
            "candidates_per_query": int(prof["candidates"] / n),
            "route_kernel_us": round(tr * 1e6, 2), "route_bytes": int(rb),
            "chain_gbs": round(chain, 1), "chain_frac": round(chain / peak, 4)}


def serve_open_loop(e8qlib, idx, mode, qn, ks, nprobes, rate_qps, seconds, seed, max_batch):
    """Open-loop Poisson arrivals through e8qlib.Server: requests of U{1..64}
    queries, k and nprobe drawn uniformly per request from `ks` / `nprobes`,
    exponential inter-arrival times at rate_qps / 32.5 requests per second;
    one thread submits on schedule, another collects. Returns the server's
    stats (latency submit -> results ready)."""
    import threading

    rng = np.random.default_rng(seed)
    req_rate = rate_qps / 32.5
    n_req = max(1, int(req_rate * seconds))
    gaps = rng.exponential(1.0 / req_rate, n_req)
    sizes = rng.integers(1, 65, n_req)
    starts = rng.integers(0, qn.shape[0] - 64, n_req)
    kreq = rng.choice(np.asarray(ks), n_req)
    npreq = rng.choice(np.asarray(nprobes), n_req)
    srv = e8qlib.Server(idx, mode=mode, max_batch=max_batch, max_k=int(max(ks)), max_nprobe=int(max(nprobes)),
                        slots=2)
    ids = []
    done = threading.Event()

    def collect():
        i = 0
        while i < n_req:
            if i < len(ids):
                srv.result(ids[i], timeout_ms=-1)
                i += 1
            else:
                time.sleep(0.0002)
        done.set()

    th = threading.Thread(target=collect)
    th.start()
    t = time.perf_counter()
    for j in range(n_req):
        t += gaps[j]
        while time.perf_counter() < t:
            pass
        ids.append(srv.submit(qn[starts[j]:starts[j] + sizes[j]], int(kreq[j]), int(npreq[j])))
    done.wait()
    th.join()
    st = srv.stats()
    srv.stop()
    st["offered_qps"] = round(rate_qps, 1)
    st["requests"] = n_req
    return st


def cpu_baseline(a, x_host, cm_host, lab_host, q_host, gt, steps=None, warmup=None):
    """The reference's own CPU search on this host, all cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    E = O.ref_module()
    if E is None:
        return None
    hc = host_cpu()
    cores = hc["cores"]
    t0 = time.perf_counter()
    ref = E.E8qIndex(a.dim, a.nbits, a.seed)
    with QuietStdout():
        ref.build(x_host, cm_host, lab_host.astype(np.uint32), num_threads=cores)
    build_s = time.perf_counter() - t0
    out = dict(hc, build_s=round(build_s, 2))
    sample = min(2048, q_host.shape[0])
    qs = q_host[:sample]
    ids, _ = ref.search(qs, a.k, a.nprobe, cores)
    out["pruned_recall"] = recall_at(ids[:gt.shape[0]], gt[:min(sample, gt.shape[0])], a.k)
    out["pruned"] = time_rounds(lambda: ref.search(qs, a.k, a.nprobe, cores), sample)
    out["pruned_qps"] = out["pruned"]["qps"]
    ref.set_disable_prune(True)
    ps = min(256, sample)
    ids_p, _ = ref.search(qs[:ps], a.k, a.nprobe, cores)
    out["plain_recall"] = recall_at(ids_p, gt[:ps], a.k)
    out["plain"] = time_rounds(lambda: ref.search(qs[:ps], a.k, a.nprobe, cores), ps, warmup=1, max_s=12.0)
    out["plain_qps"] = out["plain"]["qps"]
    ref.set_disable_prune(False)
    out["ref"] = ref
    return out


class QuietStdout:
    """Route file descriptor 1 to /dev/null (the reference's builds print
    progress lines; the bench's stdout carries one JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def me8q_cpu_baseline(xp_host, cen_host, lab_host, var_host, q_host, avg_bits, nprobe, full_n, nlist,
                      sample_n=500_000, nq=256):
    """The reference's own Me8qIndex on this host, all cores, on a bounded
    sample: the first sample_n vectors of the ME8Q workload (same lists,
    centroids and variance), its production search at nprobe over nq queries.
    The search rate in scored vectors per second is scaled to the full-size
    query (nprobe lists of full_n / nlist vectors)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    E = O.ref_module()
    if E is None:
        return None
    cores = host_cpu()["cores"]
    xs = np.ascontiguousarray(xp_host[:sample_n])
    ls = np.ascontiguousarray(lab_host[:sample_n]).astype(np.uint32)
    t0 = time.perf_counter()
    ref = E.Me8qIndex(xs.shape[1], float(avg_bits), 0)
    with QuietStdout():
        ref.build(xs, cen_host, ls, num_threads=cores, variance=var_host)
    build_s = time.perf_counter() - t0
    qs = np.ascontiguousarray(q_host[:nq])
    ref.search(qs[:16], 10, nprobe, cores)
    t0 = time.perf_counter()
    ref.search(qs, 10, nprobe, cores)
    sec = time.perf_counter() - t0
    per_list = sample_n / nlist
    vec_rate = nq * nprobe * per_list / sec
    return {"value": round(vec_rate / (nprobe * full_n / nlist), 1), "unit": "QPS", "cores": cores,
            "kind": "reference",
            "sample": (f"reference Me8qIndex(avg_bits={avg_bits}) built on the first {sample_n} vectors of this "
                       f"workload ({cores} threads, {build_s:.1f} s), production search of {nq} queries at "
                       f"nprobe {nprobe}: {vec_rate / 1e6:.1f}M scored vectors/s, scaled to a full-size query of "
                       f"{nprobe} x {full_n // nlist} vectors"),
            "sample_qps": round(nq / sec, 1), "build_s": round(build_s, 2)}


def gen_me8q(a, device):
    """ME8Q workload on `device`: z ~ N(0, diag(i^-0.8)), x = normalise(R z)
    with a seeded Haar rotation R (QR of a Gaussian); full-rank PCA (fp64
    covariance + eigh) gives the base, queries and per-dimension variance the
    index is built on; lists from 4,096 seeded rows refined by --me8q-lloyd
    Lloyd steps.
    Returns (x_raw, base_pca, q_raw, q_pca, variance, centroids, labels)."""
    import torch

    n, d, nl = a.me8q_n, a.me8q_dim, a.me8q_nlist
    g = torch.Generator(device=device)
    g.manual_seed(3000 + a.seed)
    R, _ = torch.linalg.qr(torch.randn(d, d, generator=g, device=device, dtype=torch.float64))
    sd = (torch.arange(1, d + 1, device=device, dtype=torch.float64) ** -0.4).float()
    Rf = R.float()

    def draw(m, gen):
        out = torch.empty(m, d, device=device)
        for i in range(0, m, 1 << 20):
            j = min(m, i + (1 << 20))
            z = torch.randn(j - i, d, generator=gen, device=device) * sd
            v = z @ Rf.T
            out[i:j] = v / v.norm(dim=1, keepdim=True)
        return out

    x = draw(n, g)
    gq = torch.Generator(device=device)
    gq.manual_seed(4000 + a.seed)
    q = draw(a.pool, gq)
    mean = x.double().mean(0)
    cov = torch.zeros(d, d, device=device, dtype=torch.float64)
    for i in range(0, n, 1 << 19):
        c = x[i:i + (1 << 19)].double() - mean
        cov += c.T @ c
    cov /= n
    evals, evecs = torch.linalg.eigh(cov)
    order = torch.argsort(evals, descending=True)
    V = evecs[:, order].float()
    var = evals[order].clamp_min(0).float().contiguous()
    meanf = mean.float()
    xp = torch.empty_like(x)
    for i in range(0, n, 1 << 20):
        xp[i:i + (1 << 20)] = (x[i:i + (1 << 20)] - meanf) @ V
    qp = ((q - meanf) @ V).contiguous()
    # lists: seeded rows, Lloyd steps, final assignment
    cen = xp[torch.randperm(n, generator=g, device=device)[:nl]].clone()
    lab = torch.empty(n, dtype=torch.int64, device=device)

    def assign():
        cn = (cen * cen).sum(1)
        for i in range(0, n, 1 << 18):
            blk = xp[i:i + (1 << 18)]
            lab[i:i + (1 << 18)] = torch.argmin(cn[None, :] - 2.0 * blk @ cen.T, dim=1)

    for _ in range(getattr(a, "me8q_lloyd", 3)):
        assign()
        acc = torch.zeros(nl, d, device=device, dtype=torch.float64)
        for i in range(0, n, 1 << 20):
            acc.index_add_(0, lab[i:i + (1 << 20)], xp[i:i + (1 << 20)].double())
        cnt = torch.bincount(lab, minlength=nl).double()
        keep = cnt > 0
        cen[keep] = (acc[keep] / cnt[keep, None]).float()
    assign()
    return x, xp.contiguous(), q, qp, var, cen.contiguous(), lab.to(torch.int32).contiguous()


def me8q_leg(a, e8qlib, dev, local, stream):
    """ME8Q index (mixed-rate) at the ME8Q workload, for each avg_bits of
    --me8q-avg-bits: build time, recall@10 per nprobe against an FP64 brute
    force over the raw vectors (exact grouped scan and the int8 tensor-core
    precision mode, beside the IVF ceiling), device-resident QPS of both modes
    and of the reference's production FastScan cascade (pruned mode, with its
    recall) at the smallest nprobe whose precision recall is >= 0.95 (else the
    largest), single-query latency; then open-loop serving (precision mode,
    k in {10, 100}, nprobe drawn from the values >= that nprobe) on the first
    rate that meets the recall bar (else the last)."""
    import torch

    sp = stream.cuda_stream
    t0 = time.perf_counter()
    x, xp, q, qp, var, cen, lab = gen_me8q(a, dev)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    gt = ground_truth(x, q[:a.gt], 10)
    del x
    torch.cuda.empty_cache()
    n, d = xp.shape
    nl = cen.shape[0]
    nb = a.batch
    oi = torch.empty(nb, 100, dtype=torch.int32, device=dev)
    od = torch.empty(nb, 100, dtype=torch.float32, device=dev)
    nbat = max(1, a.pool // nb)
    gtl = lab.long()[torch.from_numpy(gt.astype(np.int64)).to(dev)]
    qd = qp[:a.gt]
    cd = (qd * qd).sum(1, keepdim=True) + (cen * cen).sum(1)[None, :] - 2.0 * qd @ cen.T

    def recall(idx, npb, mode):
        ids = np.zeros((a.gt, 10), np.uint32)
        for i in range(0, a.gt, nb):
            b = min(nb, a.gt - i)
            idx.search_ptr(qp[i:i + b].data_ptr(), b, 10, npb, oi.data_ptr(), od.data_ptr(), mode, sp)
            torch.cuda.synchronize()
            ids[i:i + b] = oi.view(-1)[:b * 10].view(b, 10).cpu().numpy().view(np.uint32)
        return recall_at(ids, gt, 10)

    def qps(idx, npb, mode):
        def step(i):
            qi = qp[(i % nbat) * nb:(i % nbat) * nb + nb]
            return idx.search_ptr(qi.data_ptr(), nb, 10, npb, oi.data_ptr(), od.data_ptr(), mode, sp)

        for i in range(a.warmup):
            step(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launches = 0
        for i in range(a.steps):
            launches += step(a.warmup + i)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return a.steps * nb / (ms / 1000.0), ms / a.steps, launches

    rates = []
    serve_idx, serve_np = None, None
    avgs = [float(t) for t in str(a.me8q_avg_bits).split(",") if t]
    for ai, avg in enumerate(avgs):
        idx = e8qlib.Me8qIndex(d, avg, a.seed, device=local)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        idx.build_ptr(xp.data_ptr(), n, cen.data_ptr(), nl, lab.data_ptr(), var.data_ptr(), True, "", 0.0, sp)
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        idx.search_ptr(qp.data_ptr(), 1, 10, 1, oi.data_ptr(), od.data_ptr(), "precision", sp)  # proxy plane
        torch.cuda.synchronize()
        proxy_s = time.perf_counter() - t0
        sweep = []
        for npb in [int(t) for t in a.me8q_nprobes.split(",") if t]:
            probed = torch.topk(cd, min(npb, nl), dim=1, largest=False).indices
            ceiling = (gtl[:, :, None] == probed[:, None, :]).any(-1).float().mean().item()
            sweep.append({"nprobe": npb, "recall_precision": round(recall(idx, npb, "precision"), 4),
                          "recall_exact": round(recall(idx, npb, "batched"), 4), "ivf_ceiling": round(ceiling, 4)})
        ok = [r for r in sweep if r["recall_precision"] >= 0.95]
        npb = (ok[0] if ok else sweep[-1])["nprobe"]
        pq, pms, pl = qps(idx, npb, "precision")
        eq, ems, _ = qps(idx, npb, "batched")
        # the reference's own search (its FastScan cascade, Me8qIndex.search's default)
        rec_pruned = recall(idx, npb, "pruned")
        prq, prms, _ = qps(idx, npb, "pruned")
        lat = []
        for i in range(72):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            idx.search_ptr(qp[i].data_ptr(), 1, 10, npb, oi.data_ptr(), od.data_ptr(), "precision", sp)
            s1.record(stream)
            torch.cuda.synchronize()
            if i >= 8:
                lat.append(s0.elapsed_time(s1))
        rates.append({"avg_bits": avg, "plan": [list(p) for p in idx.plan], "bits_per_dim": round(idx.bits_per_dim, 3),
                      "memory_bytes": idx.memory_bytes, "build_s": round(build_s, 2),
                      "proxy_build_s": round(proxy_s, 2), "recall_sweep": sweep, "nprobe": npb,
                      "recall_at_10": [r["recall_precision"] for r in sweep if r["nprobe"] == npb][0],
                      "qps": round(pq, 1), "ms_per_step": round(pms, 3), "gpu_launches": int(pl),
                      "exact_qps": round(eq, 1), "exact_ms_per_step": round(ems, 3),
                      "pruned_qps": round(prq, 1), "pruned_ms_per_step": round(prms, 3),
                      "recall_pruned": round(rec_pruned, 4),
                      "single_query_ms": round(statistics.median(lat), 4)})
        if serve_idx is None and (ok or ai == len(avgs) - 1):
            serve_idx, serve_np = idx, npb
            rates[-1]["served"] = True
        else:
            del idx
        torch.cuda.empty_cache()
    xp_host = None if a.no_cpu_baseline else xp[:500_000].cpu().numpy()
    del xp
    torch.cuda.empty_cache()
    serving = None
    if not a.no_serve and serve_idx is not None:
        qh = torch.empty(a.pool, d, dtype=torch.float32, pin_memory=True)
        qh.copy_(qp.cpu())
        qn = qh.numpy()
        grid = [p for p in (16, 32, 64, 128, 256, 512) if p >= serve_np] or [serve_np]
        rng = np.random.default_rng(a.seed + 11)
        # capacity of the mixed load: one ragged batch of 4,096 queries
        kk = rng.choice([10, 100], nb).astype(np.uint32)
        pp = rng.choice(grid, nb).astype(np.uint32)
        serve_idx.search_ragged(qn[:nb], kk, pp, 100, mode="precision")
        c0 = time.perf_counter()
        serve_idx.search_ragged(qn[:nb], kk, pp, 100, mode="precision")
        cap = nb / (time.perf_counter() - c0)
        loads = []
        for frac in [float(f) for f in a.serve_loads.split(",") if f]:
            st = serve_open_loop(e8qlib, serve_idx, "precision", qn, [10, 100], grid, frac * cap, a.serve_seconds,
                                 a.seed + 13, a.batch)
            loads.append({"offered_qps": st["offered_qps"], "achieved_qps": round(st["qps"], 1),
                          "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                          "max_ms": round(st["max_ms"], 3), "requests": st["requests"],
                          "mean_batch_queries": round(st["mean_batch_queries"], 1)})
        serving = {"mode": "precision", "k": [10, 100], "nprobe": grid, "mixed_batch_capacity_qps": round(cap, 1),
                   "loads": loads}
    cpu = None
    solo = int(os.environ.get("RANK", "0")) == 0 and int(os.environ.get("WORLD_SIZE", "1")) == 1
    if xp_host is not None and solo and serve_np is not None:
        served = [r for r in rates if r.get("served")][0]
        cpu = me8q_cpu_baseline(xp_host, cen.cpu().numpy(), lab.cpu().numpy(), var.cpu().numpy(),
                                qp[:a.gt].cpu().numpy(), served["avg_bits"], serve_np, n, nl)
    out = {"workload": (f"ME8Q IVF search, {n // 1000}k x {d}-d unit vectors (spectrum i^-0.8, Haar rotation, "
                        f"full-rank PCA), {nl} lists ({a.me8q_lloyd} Lloyd steps), k=10, query batch {nb}"),
           "gen_s": round(gen_s, 2), "rates": rates, "serving": serving, "cpu_baseline": cpu}
    del serve_idx, qp, q, cen, lab, var
    torch.cuda.empty_cache()
    return out


def run_sweep(a):
    """--sweep: the configurations beside the headline, each measured the way
    the bench line is (device-resident CUDA-event timing after warm-up):
      * the 1M x 960 mixture at nbits {2, 4, 6} x nprobe {16, 64, 256}:
        recall@10 of the plain and precision paths against FP64 ground truth,
        plain (one query per launch), pruned (one query per launch), batched
        and precision (batch 4096) QPS, and the plain scan's HBM fraction;
      * nbits 6, nprobe 64: the batched and precision paths at query batches
        1 ... 4096;
      * the 100k x 128 mixture of 256 lists (sigma 0.5, flat spectrum, nbits 4,
        nprobe 16): the same paths, and the reference's CPU search on this
        host's cores;
      * 1M x 768, nbits 4, nprobe 64: the batched and precision paths at
        query batches 256 ... 8192.
    One JSON line."""
    import copy

    import torch

    import e8qlib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    pk, pk_kind = peaks()
    peak = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])

    def ev_time(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def measure(b, idx, q, gt, nprobe, batches=(4096,), with_plain=True):
        row = {"nbits": b.nbits, "nprobe": nprobe}
        ng = gt.shape[0]
        qn = q[:ng].cpu().numpy()
        ids, _ = idx.search(qn, b.k, nprobe, mode="plain")
        row["recall_plain"] = round(recall_at(ids, gt, b.k), 4)
        ids, _ = idx.search(qn, b.k, nprobe, mode="precision")
        row["recall_precision"] = round(recall_at(ids, gt, b.k), 4)
        ids, _ = idx.search(qn, b.k, nprobe, mode="pruned")
        row["recall_pruned"] = round(recall_at(ids, gt, b.k), 4)
        nmax = max(max(batches), 256)
        oi = torch.empty(nmax, b.k, dtype=torch.int32, device=dev)
        od = torch.empty(nmax, b.k, dtype=torch.float32, device=dev)
        if with_plain:
            ms = ev_time(lambda: idx.search_ptr(q.data_ptr(), 256, b.k, nprobe, oi.data_ptr(), od.data_ptr(),
                                                "plain", sp), 2)
            row["plain_qps"] = round(256 / (ms / 1000.0), 1)
            idx.profile_start()
            idx.search_ptr(q[256:].data_ptr(), 64, b.k, nprobe, oi.data_ptr(), od.data_ptr(), "plain", sp)
            torch.cuda.synchronize()
            pr = plain_roofline(idx.profile_stop(), b, peak, pk_kind)
            row["plain_scan_frac"] = pr["frac"]
            row["plain_scan_us"] = pr["launch_us"]
        for mode in ("batched", "precision", "pruned"):
            for nb in batches:
                reps = 5 if nb >= 256 else 20
                ms = ev_time(lambda: idx.search_ptr(q.data_ptr(), nb, b.k, nprobe, oi.data_ptr(), od.data_ptr(),
                                                    mode, sp), reps)
                key = f"{mode}_qps" if len(batches) == 1 else f"{mode}_qps_b{nb}"
                row[key] = round(nb / (ms / 1000.0), 1)
        return row

    out = {"sweep": "1M x 960 mixture (sigma 0.4, lambda_i ~ i^-0.5), k=10", "grid": [], "batch_sweep": None,
           "config1": None, "config4": None, "peak_hbm_gbs": peak, "peak_kind": pk_kind}
    b = copy.copy(a)
    b.n, b.dim, b.nlist, b.k, b.pool = 1_000_000, 960, 1024, 10, 4096
    b.spectrum, b.sigma = 0.5, 0.4
    x, cm, lab, q = gen_data(b, dev, 0)
    gt = ground_truth(x, q[:500], b.k)
    for nbits in (2, 4, 6):
        b.nbits = nbits
        idx = e8qlib.E8qIndex(b.dim, nbits, b.seed, device=0)
        idx.build_ptr(x.data_ptr(), b.n, cm.data_ptr(), b.nlist, lab.data_ptr(), 0.0, sp)
        torch.cuda.synchronize()
        for nprobe in (16, 64, 256):
            out["grid"].append(measure(b, idx, q, gt, nprobe))
        if nbits == 6:
            out["batch_sweep"] = measure(b, idx, q, gt, 64, batches=(1, 16, 64, 256, 1024, 4096), with_plain=False)
        del idx
        torch.cuda.empty_cache()
    del x, cm, lab, q
    torch.cuda.empty_cache()

    # 100k x 128, 256 lists, sigma 0.5, flat spectrum
    c = copy.copy(a)
    c.n, c.dim, c.nlist, c.k, c.nbits, c.pool, c.seed = 100_000, 128, 256, 10, 4, 4096, 0
    c.spectrum, c.sigma, c.nprobe = 0.0, 0.5, 16
    x, cm, lab, q = gen_data(c, dev, 0)
    gt = ground_truth(x, q[:1000], c.k)
    idx = e8qlib.E8qIndex(c.dim, c.nbits, c.seed, device=0)
    idx.build_ptr(x.data_ptr(), c.n, cm.data_ptr(), c.nlist, lab.data_ptr(), 0.0, sp)
    torch.cuda.synchronize()
    row = measure(c, idx, q, gt, 16, batches=(1024,))
    row["workload"] = workload_name(c)
    cb = cpu_baseline(c, x.cpu().numpy(), cm.cpu().numpy(), lab.cpu().numpy(), q.cpu().numpy(), gt)
    if cb is not None:
        row["cpu_reference"] = {"pruned_qps": round(cb["pruned_qps"], 1), "plain_qps": round(cb["plain_qps"], 1),
                                "recall_pruned": round(cb["pruned_recall"], 4), "cores": cb["cores"],
                                "cpu_model": cb["cpu_model"]}
    out["config1"] = row
    del idx, x, cm, lab, q
    torch.cuda.empty_cache()

    # 1M x 768, nbits 4: the precision path at query batches 256 ... 8192
    d4 = copy.copy(a)
    d4.n, d4.dim, d4.nlist, d4.k, d4.nbits, d4.pool, d4.seed = 1_000_000, 768, 1024, 10, 4, 8192, 0
    d4.spectrum, d4.sigma, d4.nprobe = 0.5, 0.4, 64
    x, cm, lab, q = gen_data(d4, dev, 0)
    gt = ground_truth(x, q[:500], d4.k)
    idx = e8qlib.E8qIndex(d4.dim, d4.nbits, d4.seed, device=0)
    idx.build_ptr(x.data_ptr(), d4.n, cm.data_ptr(), d4.nlist, lab.data_ptr(), 0.0, sp)
    torch.cuda.synchronize()
    row = measure(d4, idx, q, gt, 64, batches=(256, 1024, 4096, 8192), with_plain=False)
    row["workload"] = workload_name(d4)
    out["config4"] = row
    print(json.dumps(out), flush=True)


def main():
    a = parse()
    if a.sweep:
        return run_sweep(a)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    if a.impl == "reference":
        return run_reference(a, rank, world, dist)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import e8qlib

    pk, pk_kind = peaks()
    x, cm, lab, q = gen_data(a, dev, rank)
    gt = ground_truth(x, q[:a.gt], a.k)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    idx = e8qlib.E8qIndex(a.dim, a.nbits, a.seed, device=local)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx.build_ptr(x.data_ptr(), a.n, cm.data_ptr(), a.nlist, lab.data_ptr(), 0.0, sp)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0

    nb = a.batch if a.path in ("batched", "precision") else a.plain_batch
    out_ids = torch.empty(nb, a.k, dtype=torch.int32, device=dev)
    out_d = torch.empty(nb, a.k, dtype=torch.float32, device=dev)
    nbat = max(1, a.pool // nb)

    def step(i, mode, b=nb):
        qi = q[(i % nbat) * b:(i % nbat) * b + b]
        return idx.search_ptr(qi.data_ptr(), b, a.k, a.nprobe, out_ids.data_ptr(), out_d.data_ptr(),
                              mode, sp)

    # recall and distance error of the measured path on the ground-truth queries
    rec_ids = np.zeros((a.gt, a.k), np.uint32)
    rec_d = np.zeros((a.gt, a.k), np.float32)
    for i in range(0, a.gt, nb):
        b = min(nb, a.gt - i)
        idx.search_ptr(q[i:i + b].data_ptr(), b, a.k, a.nprobe, out_ids.data_ptr(), out_d.data_ptr(),
                       a.path, sp)
        torch.cuda.synchronize()
        rec_ids[i:i + b] = out_ids[:b].cpu().numpy().view(np.uint32)
        rec_d[i:i + b] = out_d[:b].cpu().numpy()
    recall = recall_at(rec_ids, gt, a.k)
    err_mean, err_p99, err_max = relerr(x, q[:a.gt], rec_ids, rec_d, a.k)

    for i in range(a.warmup):
        step(i, a.path)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(a.steps):
            launches += step(a.warmup + i, a.path)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_q = a.steps * nb * world
    value = total_q / (ms / 1000.0)

    # roofline of the dominant kernel: profiled pass (events around each scan)
    idx.profile_start()
    for i in range(min(a.steps, 4)):
        step(i, a.path)
    torch.cuda.synchronize()
    prof = idx.profile_stop()
    algo_per_launch = prof["algo_bytes"] / max(1, prof["scan_launches"])
    t_launch = prof["scan_ms"] / max(1, prof["scan_launches"]) / 1000.0
    achieved = algo_per_launch / t_launch / 1e9 if t_launch > 0 else 0.0
    peak = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    kernel = {"plain": "scan_plain_kernel", "batched": "batched_scan_kernel",
              "precision": "precision_scan_kernel"}[a.path]
    item_per_launch = prof["item_bytes"] / max(1, prof["scan_launches"])
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None, "kernel": kernel,
                "algo_bytes_per_launch": int(algo_per_launch),
                "launch_us": round(t_launch * 1e6, 2), "peak_kind": pk_kind,
                "item_bytes_per_launch": int(item_per_launch),
                "item_gbs": round(item_per_launch / t_launch / 1e9, 1) if t_launch > 0 else 0.0}
    if a.path == "plain":
        roofline["plain_scan"] = plain_roofline(prof, a, peak, pk_kind)
    step_breakdown = None
    if a.path == "precision" and prof.get("final_launches"):
        nl_ = max(1, prof["final_launches"])
        step_breakdown = {"route_group_ms": round(prof["prep_ms"] / nl_, 4),
                          "scan_ms": round(prof["scan_ms"] / max(1, prof["scan_launches"]), 4),
                          "select_rescore_ms": round(prof["final_ms"] / nl_, 4)}
    if a.path == "precision" and prof.get("final_launches"):
        # the select + rescore kernel: every fp16 proxy distance read once, C
        # exact rescores per query; reported as the roofline when it takes
        # longer than the scan
        f_bytes = prof["final_bytes"] / prof["final_launches"]
        f_t = prof["final_ms"] / prof["final_launches"] / 1000.0
        f_ach = f_bytes / f_t / 1e9 if f_t > 0 else 0.0
        final = {"kernel": "precision_select_kernel + precision_rescore_kernel", "achieved": round(f_ach, 1),
                 "frac": round(f_ach / peak, 4),
                 "algo_bytes_per_launch": int(f_bytes), "launch_us": round(f_t * 1e6, 2)}
        scan_part = {k2: roofline[k2] for k2 in ("kernel", "achieved", "frac", "algo_bytes_per_launch", "launch_us")}
        if f_t > t_launch:
            roofline.update(final)
            roofline["other_kernel"] = scan_part
        else:
            roofline["other_kernel"] = final
    if a.path == "precision":
        # the scan streams int8 proxy rows + (g1, h3) per vector of each probed
        # list and writes a 2-byte proxy distance per (query, vector) pair: its
        # binding roof is HBM. Beside it, the tensor side: int8 multiply-adds
        # (2 ops each) of every pair over the padded dimension against the int8
        # tcgen05 MMA rate measured on this GPU by the library's own probe.
        pd = (a.dim + 63) // 64 * 64
        ops = 2.0 * prof["candidates"] * pd / max(1, prof["scan_launches"])
        i8_peak = int8_peak(local)
        tops = ops / t_launch / 1e12 if t_launch > 0 else 0.0
        scan_entry = roofline if roofline["kernel"] == "precision_scan_kernel" else roofline["other_kernel"]
        scan_entry.update({"tensor_achieved_tops": round(tops, 1), "tensor_peak_tops": round(i8_peak, 1),
                           "tensor_frac": round(tops / i8_peak, 4),
                           "tensor_peak_kind": "int8 dense tcgen05 MMA rate measured in this run "
                                               "(e8qlib.tc_i8_gemm, 148 CTAs x 128x256x256 back-to-back MMAs)"})

    # e2e through the public numpy API with pinned host queries
    qh = torch.empty(a.pool, a.dim, dtype=torch.float32, pin_memory=True)
    qh.copy_(q.cpu())
    qn = qh.numpy()
    for i in range(2):
        idx.search(qn[:nb], a.k, a.nprobe, mode=a.path)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    for i in range(a.steps):
        j = i % nbat
        idx.search(qn[j * nb:(j + 1) * nb], a.k, a.nprobe, mode=a.path)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_wall_ms = (time.perf_counter() - w0) * 1000.0
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": round(total_q / (e2e_ms / 1000.0), 1), "unit": "QPS",
           "h2d_bytes_per_step": nb * a.dim * 4, "d2h_bytes_per_step": nb * a.k * 8,
           "host_wall_qps": round(total_q / (e2e_wall_ms / 1000.0), 1)}

    # the plain one-query-per-launch scan's own roofline (the streaming scan):
    # events around each routing and scan launch of 128 single queries
    if a.path != "plain":
        pq = 128
        pi = torch.empty(pq, a.k, dtype=torch.int32, device=dev)
        pdd = torch.empty(pq, a.k, dtype=torch.float32, device=dev)
        idx.search_ptr(q.data_ptr(), 16, a.k, a.nprobe, pi.data_ptr(), pdd.data_ptr(), "plain", sp)
        torch.cuda.synchronize()
        idx.profile_start()
        idx.search_ptr(q[pq:2 * pq].data_ptr(), pq, a.k, a.nprobe, pi.data_ptr(), pdd.data_ptr(), "plain", sp)
        torch.cuda.synchronize()
        pp = idx.profile_stop()
        roofline["plain_scan"] = plain_roofline(pp, a, peak, pk_kind)

    # the plain one-query-per-launch GPU scan on the same index (the drop-in
    # path the batched modes are compared against), a short device-resident run
    plain_qps = None
    if a.path != "plain":
        pb = 256
        pi = torch.empty(pb, a.k, dtype=torch.int32, device=dev)
        pdd = torch.empty(pb, a.k, dtype=torch.float32, device=dev)
        idx.search_ptr(q.data_ptr(), 32, a.k, a.nprobe, pi.data_ptr(), pdd.data_ptr(), "plain", sp)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        idx.search_ptr(q[pb:2 * pb].data_ptr(), pb, a.k, a.nprobe, pi.data_ptr(), pdd.data_ptr(), "plain", sp)
        p1.record(stream)
        torch.cuda.synchronize()
        plain_qps = pb / (p0.elapsed_time(p1) / 1000.0)

    # the reference's own search semantics (mode "pruned", E8qIndex.search's
    # default: its running-heap cascade, one warp per query) on a full batch
    pruned_qps = None
    if a.path != "plain":
        rb = min(a.batch, q.shape[0] // 2)
        ri = torch.empty(rb, a.k, dtype=torch.int32, device=dev)
        rdd = torch.empty(rb, a.k, dtype=torch.float32, device=dev)
        idx.search_ptr(q.data_ptr(), rb, a.k, a.nprobe, ri.data_ptr(), rdd.data_ptr(), "pruned", sp)
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        idx.search_ptr(q[rb:2 * rb].data_ptr(), rb, a.k, a.nprobe, ri.data_ptr(), rdd.data_ptr(), "pruned", sp)
        r1.record(stream)
        torch.cuda.synchronize()
        pruned_qps = rb / (r0.elapsed_time(r1) / 1000.0)

    # serving: open-loop Poisson load through the server at fractions of the
    # measured batch throughput
    serving = None
    if a.path != "plain" and not a.no_serve:
        serving = []
        for frac in [float(f) for f in a.serve_loads.split(",") if f]:
            st = serve_open_loop(e8qlib, idx, a.path, qn, [a.k], [a.nprobe], frac * value, a.serve_seconds,
                                 a.seed + 7, a.batch)
            serving.append({"offered_qps": st["offered_qps"], "achieved_qps": round(st["qps"], 1),
                            "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                            "max_ms": round(st["max_ms"], 3), "requests": st["requests"],
                            "mean_batch_queries": round(st["mean_batch_queries"], 1),
                            "k": [a.k], "nprobe": [a.nprobe]})
        # uneven requests: k and nprobe drawn per request
        mix_k, mix_np = [a.k, 100], sorted({16, 32, a.nprobe})
        frac = float([f for f in a.serve_loads.split(",") if f][0])
        st = serve_open_loop(e8qlib, idx, a.path, qn, mix_k, mix_np, frac * value, a.serve_seconds, a.seed + 11,
                             a.batch)
        serving.append({"offered_qps": st["offered_qps"], "achieved_qps": round(st["qps"], 1),
                        "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                        "max_ms": round(st["max_ms"], 3), "requests": st["requests"],
                        "mean_batch_queries": round(st["mean_batch_queries"], 1), "k": mix_k, "nprobe": mix_np})

    me8q = None
    if not a.no_me8q:
        me8q = me8q_leg(a, e8qlib, dev, local, stream)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        xh = x.cpu().numpy()
        cb = cpu_baseline(a, xh, cm.cpu().numpy(), lab.cpu().numpy(), q.cpu().numpy(), gt)
        if cb is not None:
            cb.pop("ref", None)
            cpu = {"value": round(cb["pruned_qps"], 1), "unit": "QPS", "cores": cb["cores"],
                   "kind": "reference",
                   "sample": (f"2048 queries of this workload through the reference E8qIndex.search "
                              f"(production pruned path, {cb['cores']} threads = physical cores), median of "
                              f"{cb['pruned']['rounds']} rounds after 3 warm-up passes; plain scan "
                              f"(set_disable_prune) on 256 queries"),
                   "p25": round(cb["pruned"]["p25"], 1), "p75": round(cb["pruned"]["p75"], 1),
                   "logical_cpus": cb["logical_cpus"], "cpu_model": cb["cpu_model"],
                   "recall_at_10": round(cb["pruned_recall"], 4),
                   "plain_qps": round(cb["plain_qps"], 1), "plain_recall_at_10": round(cb["plain_recall"], 4),
                   "build_s": cb["build_s"]}

    line = {
        "metric": "QPS@recall10>=0.95 (E8Q IVF search, 1 query batch per step)",
        "value": round(value, 1), "unit": "QPS", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("int8 tensor-core candidates + fp32 exact rescoring (u8 lattice codes)"
                  if a.path == "precision" else "fp32 (u8 lattice codes)"),
        "data": "synthetic (seeded Gaussian mixture generated on the GPU)",
        "config": {"workload": workload_name(a), "n": a.n, "dim": a.dim, "nlist": a.nlist,
                   "nbits": a.nbits, "k": a.k, "nprobe": a.nprobe, "query_batch": nb,
                   "path": a.path, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (codes %.0f MB > 126 MB)" % (idx.memory_bytes / 1e6),
                   "recall_at_10": round(recall, 4),
                   "relerr_mean": round(err_mean, 6), "relerr_p99": round(err_p99, 6),
                   "relerr_max": round(err_max, 6),
                   "plain_gpu_qps": None if plain_qps is None else round(plain_qps, 1),
                   "pruned_gpu_qps": None if pruned_qps is None else round(pruned_qps, 1),
                   "plain_scan_frac": roofline.get("plain_scan", {}).get("frac")},
        "recall_at_10": round(recall, 4), "build_s": round(build_s, 2),
        "relerr": {"mean": round(err_mean, 6), "p99": round(err_p99, 6), "max": round(err_max, 6),
                   "definition": "|D_hat - Delta| / Delta over the returned top-k, Delta = FP64 exact"},
        "clocks": clk.summary(), "gpu_launches": int(launches), "roofline": roofline,
        "e2e": e2e, "cpu_baseline": cpu,
        "plain_gpu_qps": None if plain_qps is None else round(plain_qps, 1),
        "pruned_gpu_qps": None if pruned_qps is None else round(pruned_qps, 1),
        "serving": serving, "me8q": me8q, "step_breakdown": step_breakdown,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_reference(a, rank, world, dist):
    """--impl reference: the reference's CPU search as the measured arm
    (rank 0 only under torchrun)."""
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    import torch

    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    x, cm, lab, q = gen_data(a, dev, 0)
    gt = ground_truth(x, q[:a.gt], a.k)
    xh, cmh, labh, qh = (t.cpu().numpy() for t in (x, cm, lab, q))
    del x
    cb = cpu_baseline(a, xh, cmh, labh, qh, gt)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (make -C oracle ref)"}))
        return
    ref = cb.pop("ref")
    cores = cb["cores"]
    nb = a.batch  # the same query batch as the measured arm
    nbat = max(1, a.pool // nb)
    for i in range(a.warmup):
        ref.search(qh[(i % nbat) * nb:(i % nbat + 1) * nb], a.k, a.nprobe, cores)
    t0 = time.perf_counter()
    for i in range(a.steps):
        j = (a.warmup + i) % nbat
        ref.search(qh[j * nb:(j + 1) * nb], a.k, a.nprobe, cores)
    sec = time.perf_counter() - t0
    value = a.steps * nb / sec
    line = {"impl": "reference", "metric": "QPS@recall10>=0.95 (E8Q IVF search, 1 query batch per step)",
            "value": round(value, 1), "unit": "QPS", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(sec * 1000 / a.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic (same seeded mixture)",
            "config": {"workload": workload_name(a),
                       "n": a.n, "dim": a.dim, "nlist": a.nlist, "nbits": a.nbits, "k": a.k,
                       "nprobe": a.nprobe, "query_batch": nb,
                       "arm": "reference CPU, production pruned search",
                       "recall_at_10": round(cb["pruned_recall"], 4)},
            "recall_at_10": round(cb["pruned_recall"], 4),
            "cpu_baseline": {"value": round(value, 1), "unit": "QPS", "cores": cores, "kind": "reference",
                             "logical_cpus": cb["logical_cpus"], "cpu_model": cb["cpu_model"],
                             "sample": (f"{nb} queries per step, {cores} threads (physical cores), "
                                        f"reference E8qIndex.search")},
            "e2e": {"value": round(value, 1), "unit": "QPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "plain_qps": round(cb["plain_qps"], 1), "build_s": cb["build_s"]}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
