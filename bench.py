#!/usr/bin/env python
"""Benchmark of the EagleImp hot path on B200: phasing + PBWT imputation.

Default workload -- batched uneven targets (cfg3): 20,000 reference
haplotypes x 400,000 sites over 40 Mb (1,000 founders) and 10,000 targets in
three array densities, 3,334 typed at 1 %, 3,333 at 3 % and 3,333 at 8 % of
the sites, each target missing U(0, 5 %) of its genotypes; K = 4096, beam
width 128.  Every density is its own typed-site set, hence its own phasing
reference and imputation PBWT (the reference imputes one typed-site set per
run, PBWTImputer.cpp:34-35,117-121).  ``--config cfg2`` runs the full
phase+impute configuration instead (10,000 x 100,000, 1,000 targets typed at
5 % with 2 % missing).  Synthetic seeded data of these shapes (the
reference's panels are not available here).

One step = the hot path over every target of the batch, timed as the
batched form runs it: each group's step captured once into a CUDA graph and
replayed, the groups' graphs concurrently (the eager step, every launch
enqueued from the host, is reported beside it).  Per density group, on the
group's own CUDA streams (the groups overlap on the device):
  * the imputation reference of its typed sites (haplotype-major panel,
    segment map, reference PBWT with prefix arrays);
  * phasing of its targets in batches (best haplotypes, condensed reference,
    PBWT, beam), in capacity mode -- no host round trip;
  * set-maximal matches of all its target haplotypes and dosages at every
    panel site.
The panel stays resident in HBM (as the reference keeps it in memory).

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's own
CPU implementation (compiled from its sources under oracle/_ref) on the host
cores on a sample of each group's targets.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from eimp_b200 import synth  # noqa: E402
from eimp_b200.bits import W, pack_rows, unpack_rows  # noqa: E402

CONFIG = "cfg3"
METRIC = "imputed hap x site dosages/sec"
UNIT = "dosages/s"
# targets per density group the CPU runs of the reference time (per step)
CPU_SAMPLE = {"cfg2": 200, "cfg3": 32}
# haplotypes of each CPU sample whose dosages are also checked against the
# FP64 dosage oracle (score/sum in double, not rounded to float)
PARITY_FP64_HAPS = 32
# device memory kept free beside the groups' buffers (the library's own
# staging, the graph form, allocator slack)
DEVICE_RESERVE_BYTES = 24e9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--targets", type=int, default=0, help="use only the first N targets of each group")
    ap.add_argument("--batch-targets", type=int, default=0, help="phasing batch size (0: from the memory budget)")
    ap.add_argument("--plain-targets", type=int, default=4,
                    help="targets per group timed one per call for the plain-form comparison (0: skip)")
    ap.add_argument("--serving-requests", type=int, default=24, help="requests of the serving run (0: skip)")
    ap.add_argument("--serving-rate", type=float, default=40.0, help="mean request arrivals per second (cfg2)")
    ap.add_argument("--serving-rate-windows", type=float, default=3.0,
                    help="mean request arrivals per second of the window requests on the cfg3 panel")
    ap.add_argument("--serving-slots", type=int, default=3, help="slots of the window-request server")
    ap.add_argument("--graph-steps", type=int, default=1,
                    help="time the step as CUDA-graph replays (default); 0: the eager step is the timed value")
    ap.add_argument("--qref-steps", type=int, default=5,
                    help="timed decodes of the panel's Qref haplotype section (0: skip)")
    ap.add_argument("--qref-variants", type=int, default=100000, help="panel variants of the Qref leg")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--cpu-sample-targets", type=int, default=0,
                    help="targets per group of the reference's CPU runs (0: the configuration's default)")
    ap.add_argument("--cfg4-targets", type=int, default=1024,
                    help="targets of the large-panel (cfg4) leg, one batch of its 50,000 (0: skip)")
    ap.add_argument("--cfg4-steps", type=int, default=2, help="timed steps of the cfg4 leg")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- workload
def load_workload(cfgname, ntargets=0):
    cfg = synth.CONFIGS[cfgname]
    panel, groups = synth.generate(cfg)
    if ntargets:
        groups = [synth.Targets(g.typed, np.ascontiguousarray(g.gt[:ntargets]),
                                np.ascontiguousarray(g.truth[:2 * ntargets])) for g in groups]
    return cfg, panel, groups


def imputed_count(tg, Mref):
    """Haplotype x site dosages of a target set: untyped sites and missing
    typed sites, both haplotypes (TargetImp.cpp:503)."""
    M = len(tg.typed)
    miss = int((tg.gt == 3).sum())
    return int(2 * ((Mref - M) * tg.gt.shape[0] + miss))


def sample_of(tg, n):
    return synth.Targets(tg.typed, np.ascontiguousarray(tg.gt[:n]), np.ascontiguousarray(tg.truth[:2 * n]))


def config_block(cfg, panel, groups, batches=None):
    dens = [f"{g.gt.shape[0]} at {len(g.typed)}" for g in groups]
    blk = {"workload": f"{cfg.name}: {panel.nhaps} ref haps x {panel.nsites} sites, "
                       f"{sum(g.gt.shape[0] for g in groups)} targets ({'; '.join(dens)} typed sites), "
                       f"K={cfg.K}, beam={cfg.beam}",
           "ref_haps": panel.nhaps, "sites": panel.nsites,
           "groups": [{"targets": int(g.gt.shape[0]), "typed_sites": len(g.typed),
                       "missing_frac": float((g.gt == 3).mean())} for g in groups],
           "targets": int(sum(g.gt.shape[0] for g in groups)), "K": cfg.K, "beam": cfg.beam,
           "l2": "flushed between timed steps (256 MiB write) and outputs > L2"}
    if batches is not None:
        blk["phasing_batches"] = batches
    return blk


# ---------------------------------------------------------------- reference CPU runs
class RefGroupSample:
    """The reference's own CPU path (oracle/_ref) on a sample of one density
    group's targets: Target::phase over the sample (PBWTPhaser::phaseCPU's
    OpenMP dynamic,1 loop), then PBWTImputer's set-maximal matches and
    imputeBunch over all panel sites.  The PBWTImputer -- the reference PBWT
    of the group's typed sites, which does not depend on the targets -- is
    built once; its build time is the group's fixed cost, and a whole
    group's time is that fixed cost plus the sample's time scaled to the
    group's targets (targets are independent)."""

    def __init__(self, cfg, panel, tg, n, nthreads):
        from oracle import refcore
        self.n, self.nthreads = n, nthreads
        self.N = tg.gt.shape[0]
        self.sub = sample_of(tg, n)
        self.Mref = panel.nsites
        self.M = len(tg.typed)
        self.rc = refcore.RefCore(panel, self.sub)
        self.rc.set_params(refcore.PhaseParams(K=cfg.K, beamwidth=cfg.beam))
        ph = pack_rows(self.sub.truth, W(self.M))
        t0 = time.perf_counter()
        self.imp = self.rc.imputer(ph, nthreads)
        t_build = time.perf_counter() - t0
        t0 = time.perf_counter()
        self.imp.retarget(ph, nthreads)
        self.t_fixed = max(0.0, t_build - (time.perf_counter() - t0))
        self.dos_group = imputed_count(tg, panel.nsites)
        self.dos_sample = imputed_count(self.sub, panel.nsites)

    def step(self, keep=None):
        """One timed pass over the sample: (phasing s, imputation s)."""
        t0 = time.perf_counter()
        mats, pats, dm, dp = self.rc.phase_range(0, self.n, self.nthreads)
        phased = np.zeros((2 * self.n, W(self.M)), np.uint64)
        phased[0::2], phased[1::2] = mats, pats
        t1 = time.perf_counter()
        self.imp.retarget(phased, self.nthreads)
        bits, dos = self.imp.bunch(self.Mref, self.nthreads)
        t2 = time.perf_counter()
        if keep is not None:
            keep.update(mats=mats, pats=pats, dm=dm, dp=dp, phased=phased, bits=bits, dos=dos,
                        absperm=self.imp.refpbwt()[1],
                        matches=[self.imp.matches(h) for h in range(min(2 * self.n, PARITY_FP64_HAPS))])
        return t1 - t0, t2 - t1

    def group_seconds(self, t_phase, t_imp):
        return self.t_fixed + (t_phase + t_imp) * self.N / self.n

    def close(self):
        self.imp.close()
        self.rc.close()


class quiet_stdout:
    """The reference prints progress to stdout; the JSON line must stay alone."""

    def __enter__(self):
        self.devnull = os.open(os.devnull, os.O_WRONLY)
        self.saved = os.dup(1)
        os.dup2(self.devnull, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.devnull)
        os.close(self.saved)


def cpu_samples(cfg, panel, groups, n):
    nthreads = os.cpu_count() or 1
    with quiet_stdout():
        return [RefGroupSample(cfg, panel, g, min(n, g.gt.shape[0]), nthreads) for g in groups], nthreads


def cpu_pass(samples, keeps=None):
    """One pass of the reference over every group's sample: whole-job
    dosages/s (fixed costs plus the sample scaled to each group), phased
    samples/s of the sample, seconds of CPU wall time."""
    tot_dos, tot_s, ph_s, ph_n, wall = 0, 0.0, 0.0, 0, 0.0
    with quiet_stdout():
        for i, s in enumerate(samples):
            tp, ti = s.step(keeps[i] if keeps is not None else None)
            tot_dos += s.dos_group
            tot_s += s.group_seconds(tp, ti)
            ph_s += tp * s.N / s.n
            ph_n += s.N
            wall += tp + ti
    return tot_dos / tot_s, ph_n / ph_s, wall


def cpu_baseline_block(samples, value, phased_per_s, wall, nthreads):
    desc = "; ".join(f"{s.n} of {s.N} targets at {s.M} typed sites (fixed PBWT build {s.t_fixed:.2f} s)"
                     for s in samples)
    return {"value": value, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "sample": f"per density group: {desc}; x all {samples[0].Mref} sites; the sample's phasing and "
                      f"imputation time scaled to the group's targets plus the group's fixed cost; "
                      f"{wall:.2f} s of CPU wall time",
            "phased_samples_per_sec": phased_per_s}


def run_reference_arm(args, rank):
    if rank != 0:
        return
    from oracle import refcore
    if not refcore.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libeimp_refcore.so was not built"}))
        return
    cfg, panel, groups = load_workload(args.config, args.targets)
    n = args.cpu_sample_targets or CPU_SAMPLE.get(cfg.name, 8)
    samples, nthreads = cpu_samples(cfg, panel, groups, n)
    vals, phs, walls = [], [], []
    for i in range(args.warmup + args.steps):
        v, p, w = cpu_pass(samples)
        if i >= args.warmup:
            vals.append(v)
            phs.append(p)
            walls.append(w)
    value = float(np.mean(vals))
    dos_total = sum(imputed_count(g, panel.nsites) for g in groups)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dos_total / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64/f32",
            "data": "synthetic (seeded Li-Stephens mosaics of the configuration's shape)",
            "config": config_block(cfg, panel, groups),
            "cpu_baseline": cpu_baseline_block(samples, value, float(np.mean(phs)), float(np.mean(walls)), nthreads),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "phased_samples_per_sec": float(np.mean(phs))}
    for s in samples:
        s.close()
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- parity
def imputed_mask(tg, ntgt, Mref):
    """(2*ntgt, Mref) bool: the sites TargetImp::imputeBunch writes for each
    target haplotype -- untyped sites and the target's missing typed sites
    (TargetImp.cpp:503)."""
    m = np.ones((ntgt, Mref), bool)
    m[:, tg.typed] = tg.gt[:ntgt] == 3
    return np.repeat(m, 2, axis=0)


def parity_group(gpu, ref, panel, tg, ntgt):
    """The GPU step's outputs for the first ntgt targets of a group against
    the reference's own CPU outputs for the same targets: bit-exact phased
    haplotypes, phasing dosages and imputed alleles; the largest dosage
    difference to the reference and to the FP64 oracle."""
    from oracle import restate as R
    out = {"targets": ntgt, "typed_sites": len(tg.typed)}
    out["phased_equal"] = bool(np.array_equal(gpu["mats"], ref["mats"]) and np.array_equal(gpu["pats"], ref["pats"]))
    out["phasing_dosages_equal"] = bool(np.array_equal(gpu["dm"], ref["dm"]) and np.array_equal(gpu["dp"], ref["dp"]))
    Mref = panel.nsites
    sel = imputed_mask(tg, ntgt, Mref)
    gb = unpack_rows(gpu["bits"], Mref).astype(bool)
    rb = unpack_rows(ref["bits"], Mref).astype(bool)
    out["imputed_alleles_equal"] = bool(np.array_equal(gb[sel], rb[sel]))
    out["dosage_max_abs_err"] = float(np.abs(gpu["dos"][sel] - ref["dos"][sel]).max(initial=0.0))
    worst = 0.0
    for h, m in enumerate(ref["matches"]):
        miss = np.where(tg.gt[h // 2] == 3)[0].astype(np.int64)
        _, _, imp, d64 = R.impute(m, ref["absperm"], panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss,
                                  ref["phased"][h], fp64=True)
        cov = imp.astype(bool) & (d64 >= 0)
        worst = max(worst, float(np.abs(gpu["dos"][h][cov].astype(np.float64) - d64[cov]).max(initial=0.0)))
    out["dosage_max_abs_err_fp64"] = worst
    out["fp64_haplotypes"] = len(ref["matches"])
    return out


def parity_block(per_group):
    ok = all(g["phased_equal"] and g["phasing_dosages_equal"] and g["imputed_alleles_equal"]
             and g["dosage_max_abs_err"] <= 1e-5 for g in per_group)
    return {"against": "reference CPU path (oracle/_ref) on each group's CPU sample", "dosage_tolerance": 1e-5,
            "groups": per_group, "ok": bool(ok),
            "dosage_max_abs_err_fp64": max(g["dosage_max_abs_err_fp64"] for g in per_group)}


# ---------------------------------------------------------------- roofline
def stage_bytes(g, cfg, rows):
    """Algorithmic bytes of every stage of one density group's step (the
    HBM traffic the work needs at least: each input read once, each output
    written once).  nt targets, M typed sites, Mref panel sites, nh panel
    haplotypes, K conditioning haplotypes, rows = sum of 2S+1 over the
    targets (S split sites), W(x) 64-bit words of an x-bit vector padded to
    512 bits, kw = 2*ceil(K/32) uint32 per compressed PBWT row."""
    nt, M, Mref, nh = g.nt, g.M, g.Mref, g.nhaps
    K = min(cfg.K, nh)
    kw = 2 * ((K + 31) // 32)
    kwr = 2 * ((nh + 31) // 32)
    ldb = (Mref + 63) // 64
    return {
        # Hamming counts + K-best + monos/calls: the typed panel once, genotypes,
        # best-haplotype lists and split/call lists written
        "prep": nh * W(M) * 8 + nt * M + nt * K * 4 + nt * M * 4 * 2 + nt * W(M) * 8,
        # condensed reference: the typed panel once, genotypes, rows written
        "cref": nh * W(M) * 8 + nt * M + rows * W(K) * 8,
        # forward + backward PBWT: condensed rows read twice, compressed rows
        # and zero counts written in both directions
        "pbwt": 2 * rows * W(K) * 8 + 2 * rows * kw * 4 + 2 * rows * 4,
        # beam: both PBWT directions, zero counts, genotypes in; phased
        # haplotypes and dosages out
        "beam": 2 * rows * kw * 4 + rows * 4 + nt * (M + 2 * W(M) * 8 + 2 * M * 4),
        # imputation reference: panel transposed (read + written), typed rows
        # read, compressed rows and prefix arrays written
        "refbuild": 2 * Mref * W(nh) * 8 + M * W(nh) * 8 + M * kwr * 4 + 4 * (M + 1) * nh,
        # matches: compressed reference rows, phased haplotypes and genotypes in
        "smm": M * kwr * 4 + 2 * nt * W(M) * 8 + nt * M,
        # dosages + alleles out, the haplotype-major panel once
        "dosage": 2 * nt * Mref * 4 + 2 * nt * ldb * 8 + nh * W(Mref) * 8,
    }


def profile_stages(groups, cfg, flush, stream_main):
    """Each group alone, stage by stage, timed with CUDA events on the
    library's stream (the phasing stages through eimp_phase_stage_ms, summed
    over the batches); the imputation reference build by wall clock around a
    synchronised call.  Outside the timed region."""
    import torch
    ms = {k: 0.0 for k in ("prep", "cref", "pbwt", "beam", "refbuild", "smm", "dosage")}
    by = {k: 0 for k in ms}
    st5 = (C.c_float * 5)()
    for g in groups:
        for k, v in stage_bytes(g, cfg, sum(g.rows)).items():
            by[k] += v
        g.ctx.synchronize()
        with torch.cuda.stream(stream_main):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.set_reference()
        g.ctx.synchronize()
        ms["refbuild"] += (time.perf_counter() - t0) * 1e3
        g.ctx.check(g.L.eimp_set_timing(g.h, 1))
        for b0, b1 in g.batches:
            g.ctx.check(g.L.eimp_phase_targets_dev(
                g.h, C.byref(g.pc), b1 - b0, g.d_gt[b0:b1].data_ptr(), g.d_mats[b0:b1].data_ptr(),
                g.d_pats[b0:b1].data_ptr(), g.d_pdm[b0:b1].data_ptr(), g.d_pdp[b0:b1].data_ptr(),
                g.d_tc[b0:b1].data_ptr(), g.d_nc[b0:b1].data_ptr()))
            g.ctx.check(g.L.eimp_phase_stage_ms(g.h, st5, 5))
            ms["prep"] += st5[0]
            ms["cref"] += st5[2]
            ms["pbwt"] += st5[3]
            ms["beam"] += st5[4]
        g.ctx.check(g.L.eimp_set_timing(g.h, 0))
        with torch.cuda.stream(g.stream):
            g.d_ph[:, 0].copy_(g.d_mats)
            g.d_ph[:, 1].copy_(g.d_pats)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(g.stream)
        g.ctx.check(g.L.eimp_imp_prepare_dev(g.h, g.nt, g.d_ph.data_ptr(), g.d_gt.data_ptr(), 0, 0, 0))
        e[1].record(g.stream)
        g.ctx.check(g.L.eimp_imp_bunch_dev(g.h, 0, g.Mref, g.d_bits.data_ptr(), g.ldb, g.d_dos.data_ptr(), g.Mref))
        e[2].record(g.stream)
        g.ctx.synchronize()
        ms["smm"] += e[0].elapsed_time(e[1])
        ms["dosage"] += e[1].elapsed_time(e[2])
    return ms, by


# ---------------------------------------------------------------- GPUEngine
# The reference's own GPU form of this call (GPUEngine::runCrefPBWTKernel:
# crefTKernel + pbwtPartedKernel) is not run: compiled for sm_100a, it ran
# for the whole 30-minute limit of a B200 call on the 5-target golden case
# (K = 64) without finishing, after every other GPU test had passed in
# seconds, so it is kept off the GPUs of this pool.
REFERENCE_GPU_ENGINE = {"unavailable": "the reference's GPU engine (crefTKernel + pbwtPartedKernel for sm_100a) "
                                       "did not finish the 5-target golden case within a 30-minute B200 call; "
                                       "it is not run on this pool"}


# ---------------------------------------------------------------- cfg4
def cfg4_fp64(g, P, typed, nhap_sample=8, frac=0.01, seed=4):
    """The cfg4 leg's FP32 dosages against the FP64 dosage oracle
    (oracle/restate.py impute_fp64_sites) on a 1 % sample of the untyped
    sites, for the first target haplotypes: their matches, the prefix-array
    slices the covering matches need and the panel rows of the sampled sites
    come from the device; the 16 GB of prefix arrays stay there."""
    import torch
    from oracle import restate as R
    rng = np.random.default_rng(seed)
    untyped = np.setdiff1d(np.arange(P.nsites), typed)
    sites = np.sort(rng.choice(untyped, max(1, int(frac * P.nsites)), replace=False)).astype(np.int64)
    d_sites = torch.from_numpy(sites).to(P.d_site.device)
    rows = P.d_site[d_sites].cpu().numpy().view(np.uint64)
    af = P.d_af.cpu().numpy()
    nh = min(nhap_sample, 2 * g.nt)
    dos = g.d_dos[:nh][:, d_sites].cpu().numpy()
    cache = {}

    def prefix_slice(en, rs, re):
        k = (en, rs, re)
        if k not in cache:
            out = np.empty(re - rs + 1, np.int32)
            g.ctx.check(g.L.eimp_imp_prefix_slice(g.h, en, rs, re, out.ctypes.data))
            cache[k] = out.astype(np.int64)
        return cache[k]

    def site_bits(j, refs):
        return (rows[j][refs >> 6] >> (refs & 63).astype(np.uint64)) & np.uint64(1)

    err, bad, cov, conf_ok, t0 = 0.0, 0, 0, True, time.perf_counter()
    for h in range(nh):
        n = C.c_size_t(0)
        g.ctx.check(g.L.eimp_imp_matches(g.h, h, None, 0, C.byref(n)))
        m = np.zeros((n.value, 4), np.int32)
        if n.value:
            g.ctx.check(g.L.eimp_imp_matches(g.h, h, m.ctypes.data, n.value, C.byref(n)))
        d64 = R.impute_fp64_sites(m, sites, typed, af, P.nhaps, prefix_slice, site_bits)
        c = d64 >= 0
        conf_ok = conf_ok and bool(np.all(dos[h][~c] == -1.0))
        if c.any():
            err = max(err, float(np.max(np.abs(dos[h][c].astype(np.float64) - d64[c]))))
            bad += int(np.count_nonzero(dos[h][c] != d64[c].astype(np.float32)))
            cov += int(c.sum())
    return {"haplotypes": nh, "sites": int(sites.size), "sample": f"{frac:.0%} of the panel sites, untyped, seeded",
            "covered": cov, "max_abs_err": err, "not_equal_to_rounded_fp64": bad,
            "uncovered_marked_conflict": conf_ok, "prefix_slices": len(cache),
            "check_s": round(time.perf_counter() - t0, 2)}


def cfg4_leg(args, local, dev):
    """The large panel (cfg4): 200,000 reference haplotypes x 1,000,000 sites
    over 60 Mb (5,000 founders, 1/x SFS down to MAF 5e-6) generated and kept
    on the device, 25 GB site-major; targets typed at 2 % (20,000 sites) with
    1 % missing, K = 8,192, beam 128.  A step is one batch of the 50,000
    targets: the imputation reference of the typed sites (the library's
    haplotype-major copy of the panel, the 20,000 x 200,000 reference PBWT
    with 16 GB of prefix arrays), phasing, matches and dosages at all
    1,000,000 sites.  Device-resident (no host copies in the timed region)."""
    import torch
    from eimp_b200 import synth, synth_device
    from eimp_b200.batch import DensityGroup
    from eimp_b200.engine import Context, PhaseParams
    cfg = synth.CONFIGS["cfg4"]
    t0 = time.perf_counter()
    gctx = Context(local)
    P = synth_device.generate(cfg, local, gctx)
    typed, gt = synth_device.targets(P, cfg.groups[0], args.cfg4_targets, seed=cfg.seed + 1)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    params = PhaseParams(K=cfg.K, beamwidth=cfg.beam)
    g = DensityGroup(local, P.d_site, P.d_af, cfg.nhaps, typed, None, None, P.cm[typed].astype(np.float32), gt,
                     params, batch_targets=args.cfg4_targets)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    g.enqueue()
    g.ctx.synchronize()
    times = []
    for _ in range(max(1, args.cfg4_steps)):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(g.stream)
        g.enqueue()
        e1.record(g.stream)
        g.ctx.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.mean(times))
    # a batch with the imputation reference already resident (the reference
    # PBWT of the typed sites is built once for all 50,000 targets)
    rtimes = []
    for _ in range(max(1, args.cfg4_steps)):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(g.stream)
        g.phase()
        g.impute()
        e1.record(g.stream)
        g.ctx.synchronize()
        rtimes.append(e0.elapsed_time(e1))
    ms_res = float(np.mean(rtimes))
    free_b, tot_b = torch.cuda.mem_get_info(dev)
    fp = cfg4_fp64(g, P, typed)
    sms, sby = profile_stages([g], cfg, flush, torch.cuda.current_stream())
    stages = {k: {"ms": sms[k], "algorithmic_bytes": sby[k], "achieved_gbs": sby[k] / (sms[k] / 1e3) / 1e9}
              for k in sms if sms[k] > 0}
    out = {"workload": f"cfg4: {cfg.nhaps} ref haps x {cfg.nsites} sites, {g.nt} of {cfg.groups[0].ntargets} "
                       f"targets (one batch) at {g.M} typed sites, K={cfg.K}, beam={cfg.beam}",
           "metric": METRIC, "unit": UNIT, "value": g.imputed() / (ms / 1e3), "ms_per_step": ms,
           "steps": len(times), "targets": g.nt, "imputed_per_step": g.imputed(),
           "phased_samples_per_sec": g.nt / (ms / 1e3), "generate_s": round(gen_s, 1),
           "batch_ms_reference_resident": ms_res}
    # the whole job: the reference built once, then every batch of the 50,000
    ntj = cfg.groups[0].ntargets
    job_s = (sms["refbuild"] + ntj / g.nt * ms_res) / 1e3
    out.update({
           "job_estimate": {"targets": ntj, "batches": -(-ntj // g.nt), "seconds": job_s,
                            "value": g.imputed() / g.nt * ntj / job_s,
                            "form": "reference build once + batches with the reference resident"},
           "device_gb_in_use": round((tot_b - free_b) / 1e9, 1), "stages": stages, "fp64": fp,
           "data": "synthetic, generated on the device (eimp_b200/synth_device.py)",
           "l2": "flushed between timed steps (256 MiB write)"})
    g.close()
    gctx.close()
    del P, g, flush
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- our arm
def max_over_ranks(x, world, dev):
    """The largest value of x over the ranks (every rank calls this at the
    same point); x itself on one GPU."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def phase_batch_targets(cfg, tgroups, Mref, nh, free_bytes):
    """Targets per phasing batch of each density group.  A batch's condensed
    references and PBWTs take about 0.25*M condensed rows per target (S ~
    0.12 M split sites at ~11 % heterozygous sites) of W(K) words plus two PBWT
    directions, and the per-target prep vectors.  Every group phases all its
    targets in one batch when those rows fit the device memory left after the
    groups' fixed buffers (dosages and imputed alleles of all sites, the
    imputation reference, the beam arenas of the resident warps); otherwise
    each group gets a share of it in proportion to its need."""
    K = min(cfg.K, nh)
    kw = 2 * ((K + 31) // 32)
    ldb = (Mref + 63) // 64
    need, fixed = [], 0.0
    for tg in tgroups:
        nt, M = tg.gt.shape
        need.append(nt * (0.25 * M * (W(K) * 8 + 2 * kw * 4 + 8) + 20.0 * M))
        fixed += 2 * nt * (Mref * 4 + ldb * 8)                                  # dosages, alleles
        fixed += nh * ldb * 8 + 4.0 * (M + 1) * nh + M * 2 * ((nh + 31) // 32) * 4   # imputation reference
        fixed += 2.5e9                                                          # beam arenas, prep vectors
    budget = max(0.0, free_bytes - fixed - DEVICE_RESERVE_BYTES)
    scale = min(1.0, budget / max(1.0, sum(need)))
    return [int(max(64, min(tg.gt.shape[0], tg.gt.shape[0] * scale))) for tg in tgroups]


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from eimp_b200.batch import DensityGroup, enqueue_step
    from eimp_b200.engine import PhaseParams
    cfg, panel, tgroups = load_workload(args.config, args.targets)
    Mref, nh_ref = panel.nsites, panel.nhaps
    dev = torch.device("cuda", local)
    main_stream = torch.cuda.current_stream(dev)

    def todev(a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            a = a.view(np.int64)
        return torch.from_numpy(a).to(dev)

    d_full = todev(panel.sitemajor)          # resident panel (referenceFullT)
    d_af = todev(panel.af.astype(np.float32))
    params = PhaseParams(K=cfg.K, beamwidth=cfg.beam)
    groups = []
    free_b, _tot = torch.cuda.mem_get_info(dev)
    bsizes = phase_batch_targets(cfg, tgroups, Mref, nh_ref, free_b)
    for tg, bauto in zip(tgroups, bsizes):
        hm, sm, cm = synth.typed_views(panel, tg.typed)
        B = args.batch_targets or bauto
        groups.append(DensityGroup(local, d_full, d_af, nh_ref, tg.typed, hm, sm, cm, tg.gt, params, B))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    # launch shapes tuned on every group's own data (eimp_b200/autotune.py)
    tuning = None
    if not args.no_autotune:
        from eimp_b200.autotune import tune_group, tune_step_shares
        tuning = {"groups": [tune_group(g) for g in groups]}
        if len(groups) > 1:
            tuning["step_beam_shares"] = tune_step_shares(groups, reps=2)

    def step_timed(graphs=False):
        e0, e1 = ev(), ev()
        e0.record(main_stream)
        for e in enqueue_step(groups, e0, capture_graphs=graphs):
            main_stream.wait_event(e)
        e1.record(main_stream)
        return e0, e1

    def timed(graphs, steps):
        """steps timed steps (L2 flushed before each); the sum of their device
        times, the largest over the ranks"""
        evs = []
        for _ in range(steps):
            flush.zero_()
            evs.append(step_timed(graphs))
        torch.cuda.synchronize()
        for g in groups:
            g.ctx.synchronize()   # status check (capacity errors would surface here)
        tot = float(np.sum([a.elapsed_time(b) for a, b in evs]))
        if world > 1:
            t = torch.tensor([tot], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
            dist.barrier()
        return tot

    # the eager step (every launch enqueued from the host), then the step as
    # the batched form runs it: each group's step captured once into a CUDA
    # graph and replayed, the groups' graphs concurrently -- the timed value
    for _ in range(args.warmup):
        enqueue_step(groups)
    for g in groups:
        g.ctx.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = sum(g.ctx.launches for g in groups)
    eager_ms = timed(False, args.steps)
    launches = sum(g.ctx.launches for g in groups) - launches0
    use_graphs = args.graph_steps > 0
    graph = None
    if use_graphs:
        ref_out = [(g.d_dos.clone(), g.d_bits.clone(), g.d_mats.clone(), g.d_pats.clone()) for g in groups]
        for g in groups:
            g.ctx.synchronize()
            g.capture()
        for _ in range(args.warmup):
            enqueue_step(groups, capture_graphs=True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    tot_ms = timed(True, args.steps) if use_graphs else eager_ms
    clocks = sampler.stop()
    if use_graphs:
        same = all(torch.equal(a, b) for g, r in zip(groups, ref_out)
                   for a, b in zip(r, (g.d_dos, g.d_bits, g.d_mats, g.d_pats)))
        del ref_out
    dos_per_step = sum(g.imputed() for g in groups)
    batches_info = [len(g.batches) for g in groups]
    targets_total = sum(g.nt for g in groups)
    value = world * dos_per_step * args.steps / (tot_ms / 1e3)
    ms_per_step = tot_ms / args.steps
    eager = {"value": world * dos_per_step * args.steps / (eager_ms / 1e3), "unit": UNIT,
             "ms_per_step": eager_ms / args.steps, "steps": args.steps,
             "form": "every launch enqueued from the host, the groups on their own streams"}
    if use_graphs:
        graph = {"value": value, "unit": UNIT, "ms_per_step": ms_per_step, "steps": args.steps,
                 "equal_to_eager": bool(same), "graphs": len(groups), "rows_reserved": [max(g.rows) for g in groups],
                 "form": "the timed step: one CUDA graph per group (capacity-mode phasing), replayed concurrently"}

    # the last timed step's outputs for each group's CPU sample (compared with
    # the reference's own outputs once the CPU runs are done)
    n_cpu = args.cpu_sample_targets or CPU_SAMPLE.get(cfg.name, 8)
    gpu_out = []
    for g in groups:
        n = min(n_cpu, g.nt)
        gpu_out.append({"bits": g.d_bits[:2 * n].cpu().numpy().view(np.uint64), "dos": g.d_dos[:2 * n].cpu().numpy(),
                        "mats": g.d_mats[:n].cpu().numpy().view(np.uint64),
                        "pats": g.d_pats[:n].cpu().numpy().view(np.uint64),
                        "dm": g.d_pdm[:n].cpu().numpy(), "dp": g.d_pdp[:n].cpu().numpy()})

    # ---- roofline: every stage alone (algorithmic bytes / its device time),
    # the dominant kernel (the beam) as the line's roofline, and the step as a
    # whole (all stages' bytes over the timed step)
    peak, peak_kind = measured_peak_hbm()
    st_ms, st_by = profile_stages(groups, cfg, flush, main_stream)
    stages = {k: {"ms": st_ms[k], "algorithmic_bytes": int(st_by[k]),
                  "achieved_gbs": st_by[k] / (st_ms[k] / 1e3) / 1e9 if st_ms[k] > 0 else None,
                  "frac": st_by[k] / (st_ms[k] / 1e3) / 1e9 / peak if st_ms[k] > 0 else None} for k in st_ms}
    stages["beam"]["phased_samples_per_sec"] = sum(g.nt for g in groups) / (st_ms["beam"] / 1e3)
    step_bytes = int(sum(st_by.values()))
    rows_total = sum(sum(g.rows) for g in groups)
    beam_ms = st_ms["beam"]
    achieved = st_by["beam"] / (beam_ms / 1e3) / 1e9
    # DRAM bytes of the beam kernel from an ncu capture of a 64-target cfg2
    # launch (160.9 MB read + 14.5 MB written), scaled by condensed rows (the
    # PBWT rows the kernel streams): those 64 targets have 71,310 rows
    traffic = 175.5e6 * rows_total / 71310.0
    roofline = {"kernel": "beam_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": st_by["beam"], "avg_launch_ms": beam_ms,
                "note": "latency-bound: one warp per target walks the beam sequentially; all batches of all groups",
                "step": {"algorithmic_bytes": step_bytes, "ms": ms_per_step,
                         "achieved_gbs": step_bytes / (ms_per_step / 1e3) / 1e9,
                         "frac": step_bytes / (ms_per_step / 1e3) / 1e9 / peak},
                "stages": stages}

    serving = None


    # ---- the plain drop-in form: one target per call (phase, matches,
    # dosages), device-resident inputs, a few targets of every group
    plain = None
    if rank == 0 and args.plain_targets > 0:
        pl_ms, pl_dos, npl_all = 0.0, 0, 0
        for g, tg in zip(groups, tgroups):
            npl = min(args.plain_targets, g.nt)
            L, h = g.L, g.h
            ep = [ev() for _ in range(2)]
            g.ctx.synchronize()
            ep[0].record(g.stream)
            for i in range(npl):
                g.ctx.check(L.eimp_phase_targets_dev(h, C.byref(g.pc), 1, g.d_gt[i:i + 1].data_ptr(),
                                                     g.d_mats[i:i + 1].data_ptr(), g.d_pats[i:i + 1].data_ptr(),
                                                     g.d_pdm[i:i + 1].data_ptr(), g.d_pdp[i:i + 1].data_ptr(),
                                                     g.d_tc[i:i + 1].data_ptr(), g.d_nc[i:i + 1].data_ptr()))
                with torch.cuda.stream(g.stream):
                    g.d_ph[i, 0].copy_(g.d_mats[i])
                    g.d_ph[i, 1].copy_(g.d_pats[i])
                g.ctx.check(L.eimp_imp_prepare_dev(h, 1, g.d_ph[i].data_ptr(), g.d_gt[i:i + 1].data_ptr(), 0, 0, 0))
                g.ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, g.d_bits[2 * i:2 * i + 2].data_ptr(), g.ldb,
                                                 g.d_dos[2 * i:2 * i + 2].data_ptr(), Mref))
            ep[1].record(g.stream)
            g.ctx.synchronize()
            pl_ms += ep[0].elapsed_time(ep[1])
            pl_dos += imputed_count(sample_of(tg, npl), Mref)
            npl_all += npl
        pl_value = pl_dos / (pl_ms / 1e3)
        plain = {"value": pl_value, "unit": UNIT, "targets": npl_all, "ms_per_target": pl_ms / npl_all,
                 "batched_over_plain": (value / world) / pl_value,
                 "form": "one target per call: eimp_phase_targets_dev, eimp_imp_prepare_dev, eimp_imp_bunch_dev"}

    # ---- the panel's Qref haplotype section (qref_spec.md section I)
    # decoded on the device into site-major rows, on the panel's first
    # variants: the section already in HBM (value), and through the host API
    # from host memory (index walk, one copy, decode); the reference's own
    # decoder on one host core beside it
    qref = None
    if args.qref_steps > 0 and rank == 0:
        g0 = groups[0]
        L, h = g0.L, g0.h
        Mq = min(Mref, args.qref_variants)
        sec = synth.qref_section(panel.sitemajor[:Mq])
        nwq = W(nh_ref)
        offs = np.zeros(Mq, np.int64)
        assert L.eimp_qref_index(sec.ctypes.data, sec.size, Mq, nh_ref // 2, offs.ctypes.data) == 0
        d_sec = torch.zeros(sec.size + 16, dtype=torch.uint8, device=dev)
        d_sec[:sec.size].copy_(torch.from_numpy(sec))
        d_offs = torch.from_numpy(offs).to(dev)
        d_rows = torch.empty(Mq * nwq, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()

        def qcall():
            g0.ctx.check(L.eimp_qref_decode_dev(h, d_sec.data_ptr(), d_offs.data_ptr(), Mq, nh_ref // 2,
                                                d_rows.data_ptr(), nwq))
        for _ in range(3):
            qcall()
        g0.ctx.synchronize()
        qms = []
        for _ in range(args.qref_steps):
            with torch.cuda.stream(g0.stream):
                flush.zero_()
            q0, q1 = ev(), ev()
            q0.record(g0.stream)
            qcall()
            q1.record(g0.stream)
            g0.ctx.synchronize()
            qms.append(q0.elapsed_time(q1))
        q_ms = float(np.mean(qms))
        same = torch.equal(d_rows.view(Mq, nwq), d_full[:Mq].view(Mq, -1))
        sec_pin = torch.from_numpy(sec).pin_memory()
        g0.ctx.check(L.eimp_qref_decode(h, sec_pin.data_ptr(), sec.size, Mq, nh_ref // 2, d_rows.data_ptr(), nwq,
                                        None))   # the context's staging buffers reach their size
        t0 = time.perf_counter()
        g0.ctx.check(L.eimp_qref_decode(h, sec_pin.data_ptr(), sec.size, Mq, nh_ref // 2, d_rows.data_ptr(), nwq,
                                        None))
        e2e_ms = (time.perf_counter() - t0) * 1e3
        qbytes = sec.size + Mq * nwq * 8
        qref = {"variants": Mq, "haplotypes": nh_ref, "section_bytes": int(sec.size),
                "coded_variants": int(sum(1 for o in offs if int(sec[o:o + 8].view(np.uint64)[0]) > 0)),
                "value": Mq / (q_ms / 1e3), "unit": "variants/s", "ms": q_ms,
                "roofline": {"bound": "hbm", "achieved": qbytes / (q_ms / 1e3) / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": qbytes / (q_ms / 1e3) / 1e9 / peak,
                             "algorithmic_bytes_per_launch": qbytes},
                "e2e": {"value": Mq / (e2e_ms / 1e3), "unit": "variants/s", "ms": e2e_ms,
                        "h2d_bytes": int(sec.size), "d2h_bytes": 0},
                "equal_to_panel": bool(same)}
        if not args.no_cpu_baseline:
            from oracle import refcore
            if refcore.available():
                t0 = time.perf_counter()
                _, rc = refcore.qref_decode(sec, Mq, nwq)
                c_s = time.perf_counter() - t0
                qref["cpu_baseline"] = {"value": Mq / c_s, "unit": "variants/s", "cores": 1, "kind": "reference",
                                        "sample": f"the first {Mq} variants, runlengthDecode of utils.h",
                                        "ok": rc == 0}
        del d_sec, d_rows, d_offs

    # ---- end to end through the host API: pinned genotypes in, phased
    # haplotypes back to the host, phased haplotypes in again for the
    # imputation, dosages and alleles out.  Every group's chain of host calls
    # runs in its own host thread with its own pinned buffers (the library's
    # calls release the interpreter lock and each group has its own context
    # and streams), so the groups overlap on the device as in the step and a
    # group's copies overlap the others' kernels
    e2e = None
    if args.e2e_steps > 0:
        # the step's device outputs are no longer needed (parity uses the
        # snapshot above); the host API stages through the contexts' own buffers
        for g in groups:
            g.d_dos = g.d_bits = None
        torch.cuda.empty_cache()
        pin = lambda *shape, dt=torch.int64: torch.empty(shape, dtype=dt).pin_memory()  # noqa: E731
        bufs = []
        h2d = d2h = 0
        for g in groups:
            bufs.append({"gt": pin(g.nt, g.M, dt=torch.uint8), "ph": pin(g.nt, 2, g.wM), "mats": pin(g.nt, g.wM),
                         "pats": pin(g.nt, g.wM), "pdm": pin(g.nt, g.M, dt=torch.float32),
                         "pdp": pin(g.nt, g.M, dt=torch.float32), "tc": pin(g.nt, dt=torch.float32),
                         "nc": pin(g.nt, dt=torch.int32), "dos": pin(2 * g.nt, Mref, dt=torch.float32),
                         "bits": pin(2 * g.nt, W(Mref))})
            h2d += 2 * g.nt * g.M + 2 * g.nt * g.wM * 8
            d2h += 2 * g.nt * g.wM * 8 + 2 * g.nt * g.M * 4 + g.nt * 8 + 2 * g.nt * Mref * 4 + 2 * g.nt * W(Mref) * 8

        def e2e_group(g, b):
            L, h = g.L, g.h
            b["gt"].copy_(torch.from_numpy(g.gt_host))
            g.set_reference()
            for b0, b1 in g.batches:
                g.ctx.check(L.eimp_phase_targets(h, C.byref(g.pc), b1 - b0, b["gt"][b0:b1].data_ptr(),
                                                 b["mats"][b0:b1].data_ptr(), b["pats"][b0:b1].data_ptr(),
                                                 b["pdm"][b0:b1].data_ptr(), b["pdp"][b0:b1].data_ptr(),
                                                 b["tc"][b0:b1].data_ptr(), b["nc"][b0:b1].data_ptr()))
            b["ph"][:, 0].copy_(b["mats"])
            b["ph"][:, 1].copy_(b["pats"])
            g.ctx.check(L.eimp_imp_prepare(h, g.nt, b["ph"].data_ptr(), b["gt"].data_ptr(), 0, 0, 0))
            g.ctx.check(L.eimp_imp_bunch(h, 0, Mref, b["bits"].data_ptr(), b["dos"].data_ptr()))

        def e2e_step():
            from eimp_b200.batch import step_order
            errs = []

            def run(i):
                try:
                    e2e_group(groups[i], bufs[i])
                except Exception as ex:   # re-raised below
                    errs.append(ex)
            ths = [threading.Thread(target=run, args=(i,)) for i in step_order(groups)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            if errs:
                raise errs[0]

        e2e_step()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        dt = max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, world, dev)
        # the copy bandwidth the dosages meet: one pinned 1 GiB device-to-host copy
        src = torch.empty(1 << 30, dtype=torch.uint8, device=dev)
        dst = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()
        dst.copy_(src)
        c0, c1 = ev(), ev()
        c0.record(main_stream)
        dst.copy_(src, non_blocking=True)
        c1.record(main_stream)
        torch.cuda.synchronize()
        d2h_gbs = (1 << 30) / (c0.elapsed_time(c1) / 1e3) / 1e9
        del src, dst
        e2e = {"value": world * dos_per_step / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3,
               "d2h_copy_gbs": round(d2h_gbs, 1), "d2h_copy_ms_per_step": round(d2h / d2h_gbs / 1e6, 1),
               "form": "host API, one host thread per group (eimp_phase_targets per batch, eimp_imp_prepare, "
                       "eimp_imp_bunch) with its own pinned buffers, the groups overlapping on the device"}
        del bufs

    # ---- serving: continuous batching of requests of 1..256 targets of the
    # first group arriving as a Poisson stream, two slots (contexts) on this
    # device; host buffers in and out; latency from submission to result
    if rank == 0 and args.serving_requests > 0 and len(groups) == 1:
        from eimp_b200.serving import GpuSlot, Server, device_bytes_per_target, load_test
        tg = tgroups[0]
        nt, M = tg.gt.shape
        hm, sm, cm = synth.typed_views(panel, tg.typed)
        srng = np.random.default_rng(cfg.seed + 7)
        sizes = np.exp(srng.uniform(0.0, np.log(256.0), size=args.serving_requests)).astype(int).clip(1, 256)
        reqs, o = [], 0
        for sz in sizes:
            idx = (o + np.arange(sz)) % nt
            reqs.append(np.ascontiguousarray(tg.gt[idx]))
            o += sz
        slots = [GpuSlot(local, hm, sm, cm, panel.sitemajor, panel.af.astype(np.float32), tg.typed, nh_ref, params)
                 for _ in range(2)]
        bpt = device_bytes_per_target(M, Mref, min(cfg.K, nh_ref), P=cfg.beam)
        free_b, _tot = torch.cuda.mem_get_info(dev)
        srv = Server(slots, max_batch_targets=512, mem_budget=0.5 * free_b, bytes_per_target=bpt)
        srv.warmup(tg.gt[np.arange(512) % nt])   # buffers at their working size
        cnt = lambda gg: int(2 * ((Mref - M) * gg.shape[0] + (gg == 3).sum()))  # noqa: E731
        serving = load_test(srv, reqs, args.serving_rate, seed=cfg.seed, count=cnt)
        srv.close()
        serving.update({"unit": UNIT, "slots": 2, "max_batch_targets": 512,
                        "request_sizes": "log-uniform 1..256 targets", "arrivals": "Poisson"})

    # ---- serving on the resident cfg3 panel (the cfg5 workload): requests of
    # log-uniform 1..5,000 targets, typed density 1-8 %, each in a random
    # 2-10 Mb window, Poisson arrivals; every request has its own typed sites,
    # so its references are built on the device from the resident panel and
    # requests overlap on the slots (admitted by device memory); the same
    # requests one at a time on one slot beside it
    if rank == 0 and args.serving_requests > 0 and len(groups) > 1:
        from eimp_b200.serving import Server, WindowSlot, load_test, window_request_bytes
        for g in groups:   # the batch's device buffers are not needed any more
            g.close()
        groups = []
        torch.cuda.empty_cache()
        reqs = synth.window_requests(cfg, panel, args.serving_requests, seed=cfg.seed + 11)
        nb = lambda r: window_request_bytes(r, nh_ref, cfg.K, cfg.beam)  # noqa: E731
        cnt = lambda r: int(2 * ((r.hi - r.lo - len(r.typed)) * r.n + (r.gt == 3).sum()))  # noqa: E731
        slots = [WindowSlot(local, d_full, d_af, panel.cm, nh_ref, params) for _ in range(args.serving_slots)]
        big = max(reqs, key=nb)
        for sl in slots:     # buffers at their working size
            sl.run(big)
        torch.cuda.synchronize()
        free_b, _tot = torch.cuda.mem_get_info(dev)

        def serve(sl, rate):
            srv = Server(sl, merge=False, mem_budget=0.8 * free_b, request_bytes=nb)
            out = load_test(srv, reqs, rate, seed=cfg.seed + 12, count=cnt)
            srv.shutdown()
            return out

        # continuous batching over the slots, then the same requests one at a
        # time (one slot, first come first served), under the same Poisson
        # arrivals; and both saturated (all requests at once) for throughput
        served = serve(slots, args.serving_rate_windows)
        fifo = serve(slots[:1], args.serving_rate_windows)
        sat = serve(slots, 1e9)
        sat1 = serve(slots[:1], 1e9)
        for sl in slots:
            sl.close()
        served.update({"unit": UNIT, "workload": "cfg5: requests on the resident cfg3 panel",
                       "slots": args.serving_slots, "arrivals": "Poisson",
                       "request_sizes": "log-uniform 1..5000 targets, typed density U(1 %, 8 %), windows U(2, 10) Mb",
                       "request_targets": [int(r.n) for r in reqs],
                       "one_at_a_time": {"p50_ms": fifo["p50_ms"], "p99_ms": fifo["p99_ms"],
                                         "throughput": fifo["throughput"], "makespan_s": fifo["makespan_s"],
                                         "unit": UNIT, "form": "the same requests and arrivals, one slot, "
                                                               "first come first served"},
                       "saturated": {"throughput": sat["throughput"], "makespan_s": sat["makespan_s"],
                                     "one_at_a_time_throughput": sat1["throughput"],
                                     "one_at_a_time_makespan_s": sat1["makespan_s"],
                                     "form": "all requests submitted at once"}})
        serving = served

    # ---- the reference's own CPU path on each group's sample, and parity of
    # the GPU step against it
    cpu = None
    parity = None
    gpuengine = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        from oracle import refcore
        if refcore.available():
            samples, nthreads = cpu_samples(cfg, panel, tgroups, n_cpu)
            keeps = [{} for _ in samples]
            cpu_pass(samples)                       # warm-up
            v, p, w = cpu_pass(samples, keeps)
            cpu = cpu_baseline_block(samples, v, p, w, nthreads)
            parity = parity_block([parity_group(go, k, panel, tg, s.n)
                                   for go, k, tg, s in zip(gpu_out, keeps, tgroups, samples)])
            for s in samples:
                s.close()
        gpuengine = REFERENCE_GPU_ENGINE

    # ---- the large panel (cfg4) on the device, after everything above
    cfg4 = None
    if rank == 0 and world == 1 and args.cfg4_targets > 0 and args.config == CONFIG:
        for g in groups:
            g.close()
        groups = []
        del d_full, d_af
        torch.cuda.empty_cache()
        cfg4 = cfg4_leg(args, local, dev)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64/f32",
                "data": "synthetic (seeded Li-Stephens mosaics of the configuration's shape)",
                "config": dict(config_block(cfg, panel, tgroups, batches_info),
                               step_form="one CUDA graph per density group, replayed concurrently" if use_graphs
                               else "eager launches"),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": int(launches), "phased_samples_per_sec": world * targets_total / (ms_per_step / 1e3),
                "plain": plain, "serving": serving, "graph": graph, "eager": eager, "qref_decode": qref,
                "parity": parity,
                "autotune": tuning, "cfg4": cfg4, "reference_gpu_engine": gpuengine}
        print(json.dumps(line), flush=True)
    for g in groups:
        g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
