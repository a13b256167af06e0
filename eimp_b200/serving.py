"""Serving loop: continuous batching of phasing + imputation requests.

The reference runs one batch of targets per process (main.cpp: read, phase,
impute, write).  A serving deployment keeps the reference panel and its
imputation PBWT resident in HBM and answers a stream of requests, each a
batch of diploid targets (genotype bytes over the typed sites), with their
phased haplotypes and imputed dosages.

* **Slots.**  Each slot owns one library context (its own CUDA streams) with
  the phasing reference and the imputation reference (typed PBWT, prefix
  arrays, haplotype-major panel) uploaded once.  Slots run concurrently, so
  the kernels of different requests overlap on the device.
* **Continuous batching.**  When a slot is free it takes, in arrival order,
  as many queued requests as fit into one launch (at most
  ``max_batch_targets`` targets) and into the device-memory budget, whatever
  their sizes; the requests that arrive meanwhile wait for the next free
  slot.  Results are split back per request.  Per-target work is independent
  (one warp per target in phasing, one per target haplotype in imputation),
  so a request's result does not depend on what it was batched with.
* **Admission by device memory.**  Every launch reserves an estimate of its
  device bytes (``bytes_per_target`` x its targets) against ``mem_budget``;
  a launch waits until the reservations in flight leave room for it.  A
  request that could never fit is failed at submission.

``Server.submit`` returns a ``concurrent.futures.Future`` whose result is a
:class:`Result`; ``Server.latencies()`` gives the per-request latencies
(submission to completion) for p50/p99.
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .bits import W


@dataclass
class Result:
    """One request's outputs: phased haplotypes (n x W(M) words each, as
    phasedTargets), imputed allele bits (2n x W(Mref) words) and dosages
    (2n x Mref floats, -1 where no match covers a site)."""
    mats: np.ndarray
    pats: np.ndarray
    bits: np.ndarray
    dosages: np.ndarray
    batch_targets: int = 0     # targets in the launch that served it
    latency_s: float = 0.0


@dataclass
class _Request:
    gt: object                 # genotype array, or a request object for slots that take one
    future: Future
    t_submit: float
    n: int = field(init=False)

    def __post_init__(self):
        self.n = self.gt.shape[0] if isinstance(self.gt, np.ndarray) else int(self.gt.n)


class GpuSlot:
    """One slot of the server on a CUDA device: a context with the phasing
    and imputation references resident; ``run`` phases and imputes a batch."""

    def __init__(self, device: int, hapmajor, sitemajor, cm, sitemajor_full, af_full, typed, nhaps: int, params):
        from .engine import Context, PBWTImputer, Phaser
        self.ctx = Context(device)
        self.phaser = Phaser(self.ctx, hapmajor, sitemajor, cm)
        self.imputer = PBWTImputer(self.ctx, sitemajor_full, af_full, typed, sitemajor, nhaps)
        self.params = params
        self.M = sitemajor.shape[0]
        self.Mref = sitemajor_full.shape[0]
        self._bufs, self._keep = {}, {}

    def _pinned(self, name: str, rows: int, cols: int, dtype):
        """A page-locked host buffer of at least rows x cols, reused across
        launches (device-to-host copies into it run at full PCIe speed and
        touch no fresh pages)."""
        buf = self._bufs.get(name)
        if buf is None or buf.shape[0] < rows:
            import torch
            nbytes = rows * cols * np.dtype(dtype).itemsize
            t = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            self._keep[name] = t
            buf = t.numpy().view(dtype).reshape(rows, cols)
            self._bufs[name] = buf
        return buf[:rows]

    def run(self, gt: np.ndarray):
        from ._lib import ptr
        mats, pats, _dm, _dp, _tc, _nc = self.phaser.phase(self.params, gt)
        n = gt.shape[0]
        phased = np.empty((2 * n, W(self.M)), np.uint64)
        phased[0::2] = mats
        phased[1::2] = pats
        self.imputer.prepareImputation(phased, gt)
        bits = self._pinned("bits", 2 * n, W(self.Mref), np.uint64)
        dos = self._pinned("dos", 2 * n, self.Mref, np.float32)
        self.ctx.check(self.ctx.L.eimp_imp_bunch(self.ctx.h, 0, self.Mref, ptr(bits), ptr(dos)))
        return mats, pats, bits.copy(), dos.copy()

    def close(self):
        self.ctx.close()


class Server:
    """Continuous-batching request loop over ``slots`` (objects with
    ``run(gt) -> (mats, pats, bits, dosages)`` and ``close()``)."""

    def __init__(self, slots, max_batch_targets: int = 256, mem_budget: float = float("inf"),
                 bytes_per_target: float = 0.0, merge: bool = True, request_bytes=None):
        """merge: requests share launches (they must share the typed sites);
        with merge=False every launch serves one request, and the requests in
        flight overlap on the slots.  request_bytes(req) overrides the
        per-target device-memory estimate."""
        if not slots:
            raise ValueError("a server needs at least one slot")
        self.slots = list(slots)
        self.max_batch = int(max_batch_targets)
        self.mem_budget = float(mem_budget)
        self.bytes_per_target = float(bytes_per_target)
        self.merge = bool(merge)
        self.request_bytes = request_bytes
        self._q: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()
        self._reserved = 0.0
        self._stop = False
        self._lat: list[float] = []
        self._batches: list[int] = []
        self._workers = [threading.Thread(target=self._work, args=(s,), daemon=True) for s in self.slots]
        for t in self._workers:
            t.start()

    # ------------------------------------------------------------ client side
    def _bytes(self, req: _Request) -> float:
        return float(self.request_bytes(req.gt)) if self.request_bytes else self.bytes_per_target * req.n

    def submit(self, gt) -> Future:
        fut: Future = Future()
        if isinstance(gt, np.ndarray) or not hasattr(gt, "n"):
            gt = np.ascontiguousarray(gt, dtype=np.uint8)
            if gt.ndim != 2 or gt.shape[0] == 0:
                fut.set_exception(ValueError("a request is a non-empty (targets x typed sites) genotype array"))
                return fut
        need = self._bytes(_Request(gt, fut, 0.0))
        if need > self.mem_budget:
            fut.set_exception(MemoryError(
                f"request needs ~{need:.3g} B of device memory, more than the budget {self.mem_budget:.3g} B"))
            return fut
        with self._cv:
            if self._stop:
                fut.set_exception(RuntimeError("server is closed"))
                return fut
            self._q.append(_Request(gt, fut, time.perf_counter()))
            self._cv.notify_all()
        return fut

    def warmup(self, gt: np.ndarray):
        """Runs one launch of ``gt`` (typically max_batch_targets targets) on
        every slot before serving, so that the slots' device and pinned host
        buffers reach their working size up front: growing them later means
        cudaFree/cudaMalloc, which synchronise the whole device and stall the
        other slots."""
        gt = np.ascontiguousarray(gt, dtype=np.uint8)
        for s in self.slots:
            s.run(gt)

    def latencies(self) -> np.ndarray:
        with self._cv:
            return np.array(self._lat)

    def batch_sizes(self) -> list[int]:
        with self._cv:
            return list(self._batches)

    def shutdown(self):
        """Stops the workers once the queue is served; the slots stay open."""
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._workers:
            t.join()

    def close(self):
        self.shutdown()
        for s in self.slots:
            s.close()

    # ------------------------------------------------------------ scheduling
    def _take(self):
        """Requests for the next launch (called with the lock held): arrival
        order, up to max_batch targets (a larger single request goes alone),
        within the memory left; None when nothing can start now."""
        batch, n, need = [], 0, 0.0
        while self._q:
            r = self._q[0]
            if batch and (not self.merge or n + r.n > self.max_batch):
                break
            more = self._bytes(r)
            if self._reserved + need + more > self.mem_budget:
                break
            batch.append(self._q.popleft())
            n += r.n
            need += more
        return (batch, n, need) if batch else None

    def _work(self, slot):
        while True:
            with self._cv:
                # serve what is queued, closing or not; exit once closed and empty
                while True:
                    got = self._take()
                    if got or (self._stop and not self._q):
                        break
                    self._cv.wait()
                if got is None:
                    return
                batch, n, reserve = got
                self._reserved += reserve
            try:
                gt = batch[0].gt if len(batch) == 1 else np.concatenate([r.gt for r in batch])
                mats, pats, bits, dos = slot.run(gt)
                if not isinstance(mats, np.ndarray):   # a slot that keeps the result on the device
                    mats, pats, bits, dos = (np.asarray(x) for x in (mats, pats, bits, dos))
                t_done = time.perf_counter()
                off = 0
                for r in batch:
                    res = Result(mats[off:off + r.n], pats[off:off + r.n], bits[2 * off:2 * (off + r.n)],
                                 dos[2 * off:2 * (off + r.n)], batch_targets=n, latency_s=t_done - r.t_submit)
                    off += r.n
                    with self._cv:
                        self._lat.append(res.latency_s)
                    r.future.set_result(res)
            except BaseException as e:  # noqa: BLE001 -- the error goes to every request of the launch
                for r in batch:
                    if not r.future.done():
                        r.future.set_exception(e)
            finally:
                with self._cv:
                    self._reserved -= reserve
                    self._batches.append(n)
                    self._cv.notify_all()


class WindowSlot:
    """A slot for requests with their own typed sites in a window of a panel
    resident on the device (the panel is shared by all slots): per request it
    builds the phasing reference (the typed rows gathered and transposed on
    the device), phases the targets, builds the imputation reference of the
    window (haplotype-major window, segment map, reference PBWT of the typed
    sites) and imputes every site of the window."""

    def __init__(self, device: int, d_sitemajor_full, d_af, cm: np.ndarray, nhaps: int, params):
        import torch
        from .engine import Context
        self.ctx = Context(device)
        self.dev = torch.device("cuda", device)
        self.d_full, self.d_af = d_sitemajor_full, d_af
        self.wN = int(d_sitemajor_full.shape[1])
        self.cm = np.asarray(cm)
        self.nhaps = nhaps
        self.params = params
        self._bufs, self._keep = {}, {}

    def _pin(self, name: str, rows: int, cols: int, dtype):
        """A (rows, cols) view of a page-locked host buffer reused across
        requests and grown to the largest request's size (rows and columns
        change with every request's targets, typed sites and window)."""
        nbytes = rows * cols * np.dtype(dtype).itemsize
        t = self._keep.get(name)
        if t is None or t.numel() < nbytes:
            import torch
            t = torch.empty(max(nbytes, 64), dtype=torch.uint8, pin_memory=True)
            self._keep[name] = t
        return t.numpy()[:nbytes].view(dtype).reshape(rows, cols)

    def run(self, req):
        import torch
        from ._lib import ptr
        L, h = self.ctx.L, self.ctx.h
        lo, hi, M, n = req.lo, req.hi, len(req.typed), req.n
        Mw = hi - lo
        typed_abs = torch.from_numpy(lo + req.typed).to(self.dev)
        typed_rel = torch.from_numpy(np.ascontiguousarray(req.typed)).to(self.dev)
        cm_t = torch.from_numpy(self.cm[lo + req.typed].astype(np.float32)).to(self.dev)
        self._keep["req"] = (typed_abs, typed_rel, cm_t)   # in use until the calls below have run
        self.ctx.check(L.eimp_phase_set_reference_dev(h, M, self.nhaps, self.d_full.data_ptr(), self.wN,
                                                      typed_abs.data_ptr(), cm_t.data_ptr()))
        gt = np.ascontiguousarray(req.gt, np.uint8)
        mats = self._pin("mats", n, W(M), np.uint64)
        pats = self._pin("pats", n, W(M), np.uint64)
        dm = self._pin("dm", n, M, np.float32)
        dp = self._pin("dp", n, M, np.float32)
        tc = self._pin("tc", n, 1, np.float32)
        nc = self._pin("nc", n, 1, np.int32)
        p = self.params.c()
        self.ctx.check(L.eimp_phase_targets(h, C.byref(p), n, ptr(gt), ptr(mats), ptr(pats), ptr(dm), ptr(dp),
                                            ptr(tc), ptr(nc)))
        phased = self._pin("phased", 2 * n, W(M), np.uint64)
        phased[0::2], phased[1::2] = mats, pats
        self.ctx.check(L.eimp_imp_set_reference_dev(h, Mw, self.nhaps, self.d_full.data_ptr() + lo * self.wN * 8,
                                                    self.d_af.data_ptr() + lo * 4, M, typed_rel.data_ptr(), None))
        self.ctx.check(L.eimp_imp_prepare(h, n, ptr(phased), ptr(gt), 0, 0, 0))
        bits = self._pin("bits", 2 * n, W(Mw), np.uint64)
        dos = self._pin("dos", 2 * n, Mw, np.float32)
        self.ctx.check(L.eimp_imp_bunch(h, 0, Mw, ptr(bits), ptr(dos)))
        return mats.copy(), pats.copy(), bits.copy(), dos.copy()

    def close(self):
        self.ctx.close()


def window_request_bytes(req, nhaps: int, K: int, P: int = 128) -> float:
    """Device memory of one window request: its references (typed rows both
    ways, the window's haplotype-major copy, prefix arrays) and its targets
    (device_bytes_per_target over the window)."""
    M, Mw = len(req.typed), req.hi - req.lo
    refs = 2 * M * W(nhaps) * 8 + nhaps * W(Mw) * 8 + 4 * (M + 1) * nhaps + Mw * 16
    return refs + req.n * device_bytes_per_target(M, Mw, min(K, nhaps), P=P)


def device_bytes_per_target(M: int, Mref: int, K: int, P: int = 128, H: int = 100, split_fraction: float = 0.25):
    """Estimate of the device memory one target occupies during a launch:
    beam arena (haplotype-path records, probability rings, interval pool),
    condensed reference and PBWTs for about split_fraction*M split sites,
    prep vectors, match lists and the imputation outputs (2 haplotypes x Mref
    dosages and bits)."""
    NH = 4 * P + 8
    arena = NH * (80 + 4 * 128 + 8 * H * 3 + 4 * 6) + 16 * (M + 1)
    rows = 2 * int(split_fraction * M) + 1
    kw = 2 * ((K + 31) // 32)
    cref = rows * W(K) * 8 + 2 * rows * kw * 4 + rows * 4
    prep = M * (4 * 3 + 1) + W(M) * 8 * 3
    matches = 2 * (M // 4 + 64) * 16
    outputs = 2 * Mref * 4 + 2 * W(Mref) * 8
    return arena + cref + prep + matches + outputs


def percentile(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else float("nan")


def load_test(server: Server, requests, rate_per_s: float, seed: int = 0, count=None):
    """Submits ``requests`` (genotype arrays) with exponential inter-arrival
    times of mean 1/rate_per_s, waits for all, and returns latency and
    throughput figures.  ``count(gt)`` gives the units a request produces
    (e.g. imputed dosages) for the throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=len(requests))
    t0 = time.perf_counter()
    futs, t_next = [], t0
    for g, gap in zip(requests, gaps):
        t_next += gap
        d = t_next - time.perf_counter()
        if d > 0:
            time.sleep(d)
        futs.append(server.submit(g))
    res = [f.result() for f in futs]
    makespan = time.perf_counter() - t0
    lat = np.array([r.latency_s for r in res]) * 1e3
    nt = lambda g: int(g.n) if hasattr(g, "n") else int(g.shape[0])  # noqa: E731
    units = sum(count(g) for g in requests) if count else sum(nt(g) for g in requests)
    return {"requests": len(requests), "targets": int(sum(nt(g) for g in requests)),
            "rate_per_s": rate_per_s, "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
            "max_ms": float(lat.max()), "makespan_s": makespan, "throughput": units / makespan,
            "mean_batch_targets": float(np.mean([r.batch_targets for r in res]))}
