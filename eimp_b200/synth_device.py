"""Seeded synthetic panels generated on the device, for panels too large to
generate or hold on the host (cfg4: 200,000 haplotypes x 1,000,000 sites,
25 GB bit-packed).

The model is the one of :mod:`eimp_b200.synth` -- founders with a 1/x
site-frequency spectrum, Li-Stephens mosaics copied a 64-site word at a time
with the words a switch falls into merged at the switch's bit, copying errors
-- drawn from torch's CUDA generator instead of numpy's, so a configuration
generated here is not the same data as :func:`synth.generate` would give.
The panel is built in blocks of haplotypes (haplotype-major) and transposed
into the site-major layout the library takes (``referenceFullT``) by the
library's device transpose; only the site positions, the genetic map and the
typed-site choice are drawn on the host.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .bits import W

_M1 = 0x5555555555555555
_M2 = 0x3333333333333333
_M4 = 0x0F0F0F0F0F0F0F0F
_H01 = 0x0101010101010101


def popcount64(x):
    """Per-element popcount of an int64 tensor (SWAR; shifts are masked so
    the arithmetic shift of negative values does not matter)."""
    x = x - ((x >> 1) & _M1)
    x = (x & _M2) + ((x >> 2) & _M2)
    x = (x + (x >> 4)) & _M4
    return (x * _H01) >> 56


def pack_bits(bits, nw: int):
    """(r, n) bool tensor -> (r, nw) int64 words, LSB first, zero padded."""
    import torch
    r, n = bits.shape
    full = torch.zeros((r, nw * 64), dtype=torch.int64, device=bits.device)
    full[:, :n] = bits.to(torch.int64)
    sh = torch.arange(64, device=bits.device, dtype=torch.int64)
    return (full.view(r, nw, 64) << sh).sum(dim=-1)


def founders(gen, f, nfounders: int, nw: int, chunk: int = 64):
    """(F, nw) int64 founder haplotypes: allele ~ Bernoulli(f) per site."""
    import torch
    n = f.numel()
    out = torch.empty((nfounders, nw), dtype=torch.int64, device=f.device)
    for a in range(0, nfounders, chunk):
        b = min(nfounders, a + chunk)
        alle = torch.rand((b - a, n), generator=gen, device=f.device) < f[None, :]
        out[a:b] = pack_bits(alle, nw)
    return out


def mosaics(gen, Fw, cm, nhap: int, mean_seg: float, copy_err: float):
    """(nhap, nw) int64 Li-Stephens mosaics of the founders Fw (F, nw) over
    the genetic positions cm (float64 tensor, one per site): Poisson(length /
    mean_seg) switches per haplotype at uniform genetic positions (a switch
    at x takes effect from the first site at or after x) to uniformly drawn
    founders, each allele flipped with probability copy_err."""
    import torch
    dev = Fw.device
    F, nw = Fw.shape
    n = cm.numel()
    c0, c1 = float(cm[0]), float(cm[-1])
    glen = c1 - c0
    counts = torch.poisson(torch.full((nhap,), glen / mean_seg, dtype=torch.float64, device=dev),
                           generator=gen).to(torch.int64)
    total = int(counts.sum())
    hid = torch.repeat_interleave(torch.arange(nhap, device=dev), counts)
    x = c0 + torch.rand(total, generator=gen, dtype=torch.float64, device=dev) * glen
    order = torch.argsort(hid.to(torch.float64) * (2.0 * glen + 1.0) + (x - c0))
    hid, x = hid[order], x[order]
    brk = torch.searchsorted(cm, x, right=False)                      # first site of the new segment
    fid = torch.randint(0, F, (total + nhap,), generator=gen, device=dev)
    bp0 = torch.zeros(nhap + 1, dtype=torch.int64, device=dev)
    bp0[1:] = torch.cumsum(counts, 0)
    seg0 = bp0[:-1] + torch.arange(nhap, device=dev)                  # first segment of each haplotype
    # founder in effect at the first site of every word
    key = hid * (n + 1) + brk
    wkey = (torch.arange(nhap, device=dev) * (n + 1))[:, None] + 64 * torch.arange(nw, device=dev)[None, :]
    nbefore = torch.searchsorted(key, wkey.reshape(-1), right=True).view(nhap, nw) - bp0[:-1, None]
    del wkey
    founder = fid[seg0[:, None] + nbefore]
    del nbefore
    words = Fw[founder, torch.arange(nw, device=dev)[None, :]]
    del founder
    # switches inside a word, in order along each haplotype
    rank = torch.arange(total, device=dev) - bp0[hid]
    inner = (brk % 64 != 0) & (brk < n)
    for r in range(int(counts.max()) if nhap else 0):
        s = torch.nonzero(inner & (rank == r)).flatten()
        if s.numel() == 0:
            continue
        h, b = hid[s], brk[s]
        w = b >> 6
        low = (torch.ones_like(b) << (b & 63)) - 1
        fnew = fid[seg0[h] + r + 1]
        words[h, w] = (words[h, w] & low) | (Fw[fnew, w] & ~low)
    # copying errors: distinct positions, their bits summed per word (= OR), XORed in
    nerr = torch.binomial(torch.full((nhap,), float(n), device=dev),
                          torch.full((nhap,), copy_err, device=dev), generator=gen).to(torch.int64)
    eh = torch.repeat_interleave(torch.arange(nhap, device=dev), nerr)
    ep = torch.randint(0, n, (eh.numel(),), generator=gen, device=dev)
    if eh.numel():
        pk = torch.unique(eh * n + ep)
        eh, ep = pk // n, pk % n
        wk = eh * nw + (ep >> 6)
        uk, inv = torch.unique(wk, return_inverse=True)
        bits = torch.zeros(uk.numel(), dtype=torch.int64, device=dev).index_add_(0, inv, torch.ones_like(ep) << (ep & 63))
        hh, ww = uk // nw, uk % nw
        words[hh, ww] = words[hh, ww] ^ bits
    return words


@dataclass
class DevicePanel:
    """A panel resident on the device: ``d_site`` (nsites, W(nhaps)) int64
    site-major rows (``referenceFullT``), ``d_af`` float32 alternative
    allele frequencies; positions and genetic map on the host; the founders
    and the generator stay on the device to draw targets."""
    nhaps: int
    nsites: int
    pos: np.ndarray
    cm: np.ndarray
    d_site: object
    d_af: object
    d_founders: object
    d_cm: object
    gen: object
    cfg: object


def generate(cfg, device: int = 0, ctx=None, block: int = 8192) -> DevicePanel:
    """The panel of ``cfg`` (a :class:`synth.SynthConfig`) on the device."""
    import torch
    from .engine import Context
    dev = torch.device("cuda", device)
    ctx = ctx or Context(device)
    rng = np.random.default_rng(cfg.seed)
    n, nh = cfg.nsites, cfg.nhaps
    L = int(cfg.segment_mb * 1e6)
    pos = np.sort(rng.integers(0, L - n, n)) + np.arange(n)
    cm = pos.astype(np.float64) * (cfg.cm_per_mb / 1e6)
    u = rng.uniform(0.0, 1.0, n)
    f = cfg.maf_min * (0.5 / cfg.maf_min) ** u
    f = np.where(rng.uniform(0.0, 1.0, n) < 0.5, 1.0 - f, f)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(cfg.seed))
    nw, wn = W(n), W(nh)
    d_cm = torch.from_numpy(cm).to(dev)
    Fw = founders(gen, torch.from_numpy(f.astype(np.float32)).to(dev), cfg.founders, nw)
    d_site = torch.zeros((n, wn), dtype=torch.int64, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    for h0 in range(0, nh, block):
        h1 = min(nh, h0 + block)
        words = mosaics(gen, Fw, d_cm, h1 - h0, cfg.mean_segment_cm, cfg.copy_err)
        ev = torch.cuda.Event()
        ev.record()
        stream.wait_event(ev)
        # haplotypes h0..h1-1 are bits h0..h1-1 of every site row (h0 a multiple of 64)
        ctx.check(ctx.L.eimp_transpose_bits_dev(ctx.h, words.data_ptr(), h1 - h0, nw,
                                                d_site.data_ptr() + (h0 // 64) * 8, n, wn))
        ctx.synchronize()
        del words
    d_af = torch.empty(n, dtype=torch.float32, device=dev)
    step = max(1, (1 << 27) // wn)
    for s0 in range(0, n, step):
        s1 = min(n, s0 + step)
        d_af[s0:s1] = (popcount64(d_site[s0:s1]).sum(dim=1).to(torch.float64) / float(nh)).to(torch.float32)
    return DevicePanel(nh, n, pos.astype(np.int64), cm, d_site, d_af, Fw, d_cm, gen, cfg)


def targets(panel: DevicePanel, group, ntargets: int, seed: int, block: int = 8192):
    """``ntargets`` held-out mosaic targets of ``group`` (a
    :class:`synth.TargetGroup`): typed sites (int64, ascending), genotypes
    (ntargets, M) uint8 with 3 = missing, exactly round(rate * M) missing
    sites per target at the group's rate."""
    import torch
    cfg = panel.cfg
    rng = np.random.default_rng(seed)
    n = panel.nsites
    m = max(2, int(round(group.typed_frac * n)))
    typed = np.sort(rng.choice(n, m, replace=False)).astype(np.int64)
    d_typed = torch.from_numpy(typed).to(panel.d_site.device)
    tw, tb = d_typed >> 6, d_typed & 63
    th = torch.empty((2 * ntargets, m), dtype=torch.uint8, device=panel.d_site.device)
    for a in range(0, 2 * ntargets, block):
        b = min(2 * ntargets, a + block)
        words = mosaics(panel.gen, panel.d_founders, panel.d_cm, b - a, cfg.mean_segment_cm, cfg.copy_err)
        th[a:b] = ((words[:, tw] >> tb) & 1).to(torch.uint8)
        del words
    gt = (th[0::2] + th[1::2]).cpu().numpy()
    for t in range(ntargets):
        rate = rng.uniform(group.miss_lo, group.miss_hi) if group.miss_hi > group.miss_lo else group.miss_lo
        k = int(round(rate * m))
        if k:
            gt[t, rng.choice(m, k, replace=False)] = 3
    return typed, np.ascontiguousarray(gt)
