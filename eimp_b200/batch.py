"""Batched form of the hot path: many targets of several array densities.

The reference phases and imputes one target set per run, all typed at the
same sites (PBWTImputer assumes one shared typed-site set,
PBWTImputer.cpp:34-35,117-121).  A batch with several array densities is
therefore several target sets over one resident panel, each with its own
typed sites, phasing reference (the panel at those sites) and imputation
reference (the PBWT and prefix arrays of those sites).

:class:`DensityGroup` is one such set on one device.  It owns a library
context, so its work runs on its own CUDA streams and the groups of a batch
overlap on the device.  Its targets are phased in batches of at most
``batch_targets`` (the condensed references and PBWTs of a batch must fit),
in capacity mode: the rows of every batch are reserved once, so a step makes
no host round trip and the whole step is enqueued without waiting.  Then all
its target haplotypes are imputed at every panel site in one match search
and one dosage launch.  :func:`enqueue_step` starts the groups of a batch
after one event and joins them into one, so a step can be timed on the
device and captured into CUDA graphs (one per group).

Inputs and outputs stay in device memory (torch tensors); the host API
(``*_host`` methods) copies genotypes in and phased haplotypes and dosages
out.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .bits import W


def _dev_tensor(a, dev):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a).to(dev)


class DensityGroup:
    """The targets of one typed-site set on one device (see the module
    docstring).  ``d_full``/``d_af`` are the resident panel (site-major rows
    of W(nhaps) words, allele frequencies) shared by all groups."""

    def __init__(self, device: int, d_full, d_af, nhaps: int, typed: np.ndarray, hapmajor_typed,
                 sitemajor_typed, cm_typed: np.ndarray, gt: np.ndarray, params, batch_targets: int = 1024):
        import torch
        from .engine import Context, Phaser
        self.ctx = Context(device)
        self.L, self.h = self.ctx.L, self.ctx.h
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream, device=self.dev)
        self.params = params
        self.pc = params.c()
        self.nhaps = nhaps
        self.Mref = int(d_full.shape[0])
        self.typed = np.ascontiguousarray(typed, np.int64)
        self.M = len(self.typed)
        self.wM = W(self.M)
        self.ldb = (self.Mref + 63) // 64
        gt = np.ascontiguousarray(gt, np.uint8)
        self.gt_host = gt
        self.nt = gt.shape[0]
        self.d_full, self.d_af = d_full, d_af
        self.d_typed = _dev_tensor(self.typed, self.dev)
        if hapmajor_typed is None:
            # both references of the typed sites built on the device from the
            # resident panel (no host copy of the typed views)
            self.d_cm = _dev_tensor(np.asarray(cm_typed, np.float32), self.dev)
            self.ctx.check(self.L.eimp_phase_set_reference_dev(self.h, self.M, nhaps, d_full.data_ptr(),
                                                               int(d_full.shape[1]), self.d_typed.data_ptr(),
                                                               self.d_cm.data_ptr()))
            self.d_sitetyped = None
        else:
            Phaser(self.ctx, hapmajor_typed, sitemajor_typed, cm_typed)   # phasing reference, resident
            self.d_sitetyped = _dev_tensor(sitemajor_typed, self.dev)
        self.d_gt = _dev_tensor(gt, self.dev)
        nt, wM, M, Mref = self.nt, self.wM, self.M, self.Mref
        i64, f32, i32 = torch.int64, torch.float32, torch.int32
        self.d_mats = torch.empty((nt, wM), dtype=i64, device=self.dev)
        self.d_pats = torch.empty((nt, wM), dtype=i64, device=self.dev)
        self.d_pdm = torch.empty((nt, M), dtype=f32, device=self.dev)
        self.d_pdp = torch.empty((nt, M), dtype=f32, device=self.dev)
        self.d_tc = torch.empty(nt, dtype=f32, device=self.dev)
        self.d_nc = torch.empty(nt, dtype=i32, device=self.dev)
        self.d_ph = torch.empty((nt, 2, wM), dtype=i64, device=self.dev)   # phased haplotypes, mat/pat interleaved
        self.d_dos = torch.empty((2 * nt, Mref), dtype=f32, device=self.dev)
        self.d_bits = torch.empty((2 * nt, self.ldb), dtype=i64, device=self.dev)
        # batches and their condensed rows (one sizing pass on the device)
        B = max(1, min(int(batch_targets), nt))
        self.batches = [(b, min(nt, b + B)) for b in range(0, nt, B)]
        ns = np.zeros(nt, np.int32)
        for b0, b1 in self.batches:
            self.ctx.check(self.L.eimp_phase_prep(self.h, C.byref(self.pc), b1 - b0, gt[b0:b1].ctypes.data, None,
                                                  None, None, None, None, None, ns[b0:b1].ctypes.data, None))
        self.rows = [int(np.sum(2 * ns[b0:b1].astype(np.int64) + 1)) for b0, b1 in self.batches]
        self.nsplits = ns
        self.ctx.check(self.L.eimp_phase_reserve(self.h, C.byref(self.pc), B, max(self.rows)))

    # -------------------------------------------------------------- step
    def set_reference(self):
        """PBWTImputer construction for this typed-site set: haplotype-major
        panel, segment map and reference PBWT with prefix arrays, built on the
        context's side stream (overlapping the phasing that follows)."""
        self.ctx.check(self.L.eimp_imp_set_reference_dev(
            self.h, self.Mref, self.nhaps, self.d_full.data_ptr(), self.d_af.data_ptr(), self.M,
            self.d_typed.data_ptr(), None if self.d_sitetyped is None else self.d_sitetyped.data_ptr()))

    def phase(self):
        import torch
        L, h = self.L, self.h
        for b0, b1 in self.batches:
            self.ctx.check(L.eimp_phase_targets_dev(
                h, C.byref(self.pc), b1 - b0, self.d_gt[b0:b1].data_ptr(), self.d_mats[b0:b1].data_ptr(),
                self.d_pats[b0:b1].data_ptr(), self.d_pdm[b0:b1].data_ptr(), self.d_pdp[b0:b1].data_ptr(),
                self.d_tc[b0:b1].data_ptr(), self.d_nc[b0:b1].data_ptr()))
        with torch.cuda.stream(self.stream):
            self.d_ph[:, 0].copy_(self.d_mats)
            self.d_ph[:, 1].copy_(self.d_pats)

    def impute(self, setmaxerrors: int = 0, imputeCalls: int = 0):
        self.ctx.check(self.L.eimp_imp_prepare_dev(self.h, self.nt, self.d_ph.data_ptr(), self.d_gt.data_ptr(),
                                                   setmaxerrors, imputeCalls, 0))
        self.ctx.check(self.L.eimp_imp_bunch_dev(self.h, 0, self.Mref, self.d_bits.data_ptr(), self.ldb,
                                                 self.d_dos.data_ptr(), self.Mref))

    def enqueue(self):
        self.set_reference()
        self.phase()
        self.impute()

    # -------------------------------------------------------------- graph form
    def capture(self):
        """Capture one step of this group into the context's CUDA graph."""
        self.ctx.check(self.L.eimp_capture_begin(self.h))
        try:
            self.enqueue()
        finally:
            self.ctx.check(self.L.eimp_capture_end(self.h))

    def replay(self):
        self.ctx.check(self.L.eimp_graph_launch(self.h))

    # -------------------------------------------------------------- counts
    def imputed(self) -> int:
        """Haplotype x site dosages the step imputes: untyped sites and the
        targets' missing typed sites, both haplotypes."""
        return int(2 * ((self.Mref - self.M) * self.nt + int((self.gt_host == 3).sum())))

    def close(self):
        self.ctx.close()


def step_order(groups):
    """The order in which a step enqueues its groups: most condensed rows
    (phasing work) first, so that the longest chain of kernels -- the densest
    group's -- takes the SMs first and the lighter groups fill in beside it."""
    return sorted(range(len(groups)), key=lambda i: -sum(groups[i].rows))


def enqueue_step(groups, start_event=None, capture_graphs=False):
    """One step of every group: each group's stream waits for start_event
    (when given), the groups run concurrently, and the returned events (one
    per group, in the order of ``groups``, recorded at the end of its step)
    mark their ends."""
    import torch
    ends = [None] * len(groups)
    for i in step_order(groups):
        g = groups[i]
        if start_event is not None:
            g.stream.wait_event(start_event)
        if capture_graphs:
            g.replay()
        else:
            g.enqueue()
        e = torch.cuda.Event()
        e.record(g.stream)
        ends[i] = e
    return ends
