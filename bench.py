#!/usr/bin/env python
"""Benchmark of the EagleImp hot path on B200: phasing + PBWT imputation.

Default workload: the full phase+impute configuration -- 10,000 reference
haplotypes x 100,000 sites over 20 Mb (500 founders), 1,000 targets typed at
5 % of the sites with 2 % missing, K=4096, beam width 128, 95,000 imputed
sites.  Synthetic seeded data of that shape (the reference's panels are not
available here).

One step = one pass of the hot path over the batch of targets:
  phasing (stage "phase", when built): best haplotypes, condensed reference,
    PBWT, beam phasing of every target;
  imputation: reference PBWT + prefix arrays of the typed sites, set-maximal
    matches of every target haplotype, dosages of every reference site.
The panel itself stays resident in HBM (as the reference keeps it in memory).

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's own
CPU implementation (compiled from its sources under oracle/_ref) on the host
cores instead.
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
from eimp_b200.bits import W, pack_rows  # noqa: E402

CONFIG = "cfg2"
METRIC = "imputed hap x site dosages/sec"
UNIT = "dosages/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--plain-targets", type=int, default=16,
                    help="targets timed one per call for the plain-form comparison (0: skip)")
    ap.add_argument("--serving-requests", type=int, default=40, help="requests of the serving run (0: skip)")
    ap.add_argument("--graph-steps", type=int, default=3, help="replays timed in the CUDA-graph form (0: skip)")
    ap.add_argument("--qref-steps", type=int, default=5,
                    help="timed decodes of the panel's Qref haplotype section (0: skip)")
    ap.add_argument("--serving-rate", type=float, default=40.0, help="mean request arrivals per second")
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--stages", default="phase,impute", help="comma list of: phase, impute")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-targets", type=int, default=200)
    ap.add_argument("--targets", type=int, default=0, help="use only the first N targets (small profiling case)")
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
    tg = groups[0]
    if ntargets:
        tg = synth.Targets(tg.typed, np.ascontiguousarray(tg.gt[:ntargets]),
                           np.ascontiguousarray(tg.truth[:2 * ntargets]))
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    return cfg, panel, tg, hm, sm, cm


def imputed_count(tg, Mref):
    M = len(tg.typed)
    miss = (tg.gt == 3).sum(axis=1)
    return int(2 * ((Mref - M) * tg.gt.shape[0] + miss.sum()))


# ---------------------------------------------------------------- reference arm / CPU baseline
def cpu_reference_sample(cfg, panel, tg, ntgt, nthreads, stages, keep=None):
    """The reference's own CPU path (oracle/_ref) on a bounded target sample:
    phasing (PBWTPhaser::phaseCPU loop) and/or PBWTImputer prepare + bunch.
    With ``keep`` (a dict) its outputs are stored there after the timing:
    phased haplotypes and dosages, imputed alleles and dosages, and the
    matches and prefix arrays of the first haplotypes (for the FP64 oracle)."""
    from oracle import refcore
    sub = synth.Targets(tg.typed, np.ascontiguousarray(tg.gt[:ntgt]), np.ascontiguousarray(tg.truth[:2 * ntgt]))
    rc = refcore.RefCore(panel, sub)
    rc.set_params(refcore.PhaseParams(K=cfg.K, beamwidth=cfg.beam))
    M = len(tg.typed)
    t0 = time.perf_counter()
    if "phase" in stages:
        mats, pats, dm, dp = rc.phase_range(0, ntgt, nthreads)
        phased = np.zeros((2 * ntgt, W(M)), np.uint64)
        phased[0::2] = mats
        phased[1::2] = pats
    else:
        phased = pack_rows(sub.truth, W(M))
    t1 = time.perf_counter()
    dt_imp = 0.0
    imp = None
    if "impute" in stages:
        imp = rc.imputer(phased, nthreads)
        bits, dos = imp.bunch(panel.nsites, nthreads)
        dt_imp = time.perf_counter() - t1
    dt = time.perf_counter() - t0
    if keep is not None:
        keep["phased"] = phased
        if "phase" in stages:
            keep.update(mats=mats, pats=pats, dm=dm, dp=dp)
        if imp is not None:
            keep.update(bits=bits, dos=dos, absperm=imp.refpbwt()[1],
                        matches=[imp.matches(h) for h in range(min(2 * ntgt, PARITY_FP64_HAPS))])
    if imp is not None:
        imp.close()
    rc.close()
    return dt, t1 - t0, dt_imp


def cpu_port_sample(cfg, panel, tg, ntgt, nthreads, stages):
    """The oracle restatement (when the reference build is absent)."""
    from oracle import restate as R
    M = len(tg.typed)
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    t0 = time.perf_counter()
    if "phase" in stages:
        P = R.params_c(K=cfg.K, beamwidth=cfg.beam)
        mats, pats, _, _ = R.phase_many(tg.gt[:ntgt], hm, sm, cm, P, nthreads)
        phased = np.zeros((2 * ntgt, W(M)), np.uint64)
        phased[0::2] = mats
        phased[1::2] = pats
    else:
        phased = pack_rows(tg.truth[:2 * ntgt], W(M))
    t1 = time.perf_counter()
    if "impute" in stages:
        compr, c0, ap = R.pbwt(sm, panel.nhaps, absperm=True)
        for h in range(2 * ntgt):
            miss = np.where(tg.gt[h // 2] == 3)[0].astype(np.int64)
            m = R.smmatches(compr, c0, M, panel.nhaps, phased[h], miss)
            R.impute(m, ap, panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss, phased[h])
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, t2 - t1


def cpu_baseline(cfg, panel, tg, ntgt, stages, keep=None):
    nthreads = os.cpu_count() or 1
    from oracle import refcore
    kind = "reference" if refcore.available() else "port"
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)   # the reference prints progress to stdout
    try:
        if kind == "reference":
            dt, dtp, dti = cpu_reference_sample(cfg, panel, tg, ntgt, nthreads, stages, keep)
        else:
            dt, dtp, dti = cpu_port_sample(cfg, panel, tg, ntgt, nthreads if "phase" in stages else 1, stages)
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)
    sub = synth.Targets(tg.typed, tg.gt[:ntgt], tg.truth[:2 * ntgt])
    dos = imputed_count(sub, panel.nsites)
    out = {"value": dos / dt if "impute" in stages else None, "unit": UNIT, "cores": nthreads, "kind": kind,
           "sample": f"{ntgt} of {tg.gt.shape[0]} targets ({2 * ntgt} haplotypes) x all {panel.nsites} sites, "
                     f"stages {','.join(stages)}, {dt:.2f} s wall"}
    if "phase" in stages:
        out["phased_samples_per_sec"] = ntgt / dtp
    return out, dt


# haplotypes of the CPU sample whose dosages are also checked against the FP64
# dosage oracle (score/sum in double, not rounded to float)
PARITY_FP64_HAPS = 32


def imputed_mask(tg, ntgt, Mref):
    """(2*ntgt, Mref) bool: the sites TargetImp::imputeBunch writes for each
    target haplotype -- untyped sites and the target's missing typed sites
    (TargetImp.cpp:503)."""
    m = np.ones((ntgt, Mref), bool)
    m[:, tg.typed] = tg.gt[:ntgt] == 3
    return np.repeat(m, 2, axis=0)


def parity_block(gpu, ref, cfg, panel, tg, ntgt, stages):
    """Compare the GPU step's outputs for the first ntgt targets with the
    reference's own CPU outputs on the same targets (bit-exact), and state the
    largest dosage error against the reference and against the FP64 oracle."""
    from eimp_b200.bits import unpack_rows
    out = {"targets": ntgt, "against": "reference CPU path (oracle/_ref) on the CPU sample"}
    if "phase" in stages and "mats" in ref:
        out["phased_equal"] = bool(np.array_equal(gpu["mats"], ref["mats"]) and np.array_equal(gpu["pats"], ref["pats"]))
        out["phasing_dosages_equal"] = bool(np.array_equal(gpu["dm"], ref["dm"]) and np.array_equal(gpu["dp"], ref["dp"]))
    if "impute" in stages and "dos" in ref:
        Mref = panel.nsites
        sel = imputed_mask(tg, ntgt, Mref)
        gb = unpack_rows(gpu["bits"], Mref).astype(bool)
        rb = unpack_rows(ref["bits"], Mref).astype(bool)
        out["imputed_alleles_equal"] = bool(np.array_equal(gb[sel], rb[sel]))
        d = np.abs(gpu["dos"][sel] - ref["dos"][sel])
        out["dosage_max_abs_err"] = float(d.max(initial=0.0))
        out["dosage_tolerance"] = 1e-5
        from oracle import restate as R
        worst = 0.0
        for h, m in enumerate(ref["matches"]):
            miss = np.where(tg.gt[h // 2] == 3)[0].astype(np.int64)
            _, _, imp, d64 = R.impute(m, ref["absperm"], panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss,
                                      ref["phased"][h], fp64=True)
            cov = imp.astype(bool) & (d64 >= 0)
            worst = max(worst, float(np.abs(gpu["dos"][h][cov].astype(np.float64) - d64[cov]).max(initial=0.0)))
        out["dosage_max_abs_err_fp64"] = worst
        out["fp64_haplotypes"] = len(ref["matches"])
    out["ok"] = all(v for k, v in out.items() if k.endswith("_equal")) and \
        out.get("dosage_max_abs_err", 0.0) <= 1e-5
    return out


def run_reference_arm(args, rank):
    stages = args.stages.split(",")
    if rank != 0:
        return
    cfg, panel, tg, hm, sm, cm = load_workload(args.config)
    ntgt = args.cpu_sample_targets
    times = []
    res = None
    for i in range(args.warmup + args.steps):
        res, dt = cpu_baseline(cfg, panel, tg, ntgt, stages)
        if i >= args.warmup:
            times.append(dt)
    sub = synth.Targets(tg.typed, tg.gt[:ntgt], tg.truth[:2 * ntgt])
    dos = imputed_count(sub, panel.nsites)
    tot = float(np.sum(times))
    value = dos * len(times) / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64/f32",
            "data": "synthetic (seeded Li-Stephens mosaics of the configuration's shape)",
            "config": config_block(cfg, panel, tg, stages),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "phased_samples_per_sec" in res:
        line["phased_samples_per_sec"] = res["phased_samples_per_sec"]
    print(json.dumps(line), flush=True)


def config_block(cfg, panel, tg, stages):
    return {"workload": f"{cfg.name}: {panel.nhaps} ref haps x {panel.nsites} sites, {tg.gt.shape[0]} targets "
                        f"typed at {len(tg.typed)} sites, K={cfg.K}, beam={cfg.beam}",
            "stages": stages, "ref_haps": panel.nhaps, "sites": panel.nsites, "typed_sites": len(tg.typed),
            "targets": int(tg.gt.shape[0]), "K": cfg.K, "beam": cfg.beam,
            "l2": "flushed between timed steps (256 MiB write) and outputs > L2"}


# ---------------------------------------------------------------- our arm
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
    from eimp_b200.engine import Context
    stages = args.stages.split(",")
    cfg, panel, tg, hm, sm, cm = load_workload(args.config, args.targets)
    nt = tg.gt.shape[0]
    M, Mref, nh_ref = len(tg.typed), panel.nsites, panel.nhaps
    ctx = Context(local)
    L, h = ctx.L, ctx.h
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def todev(a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            a = a.view(np.int64)
        return torch.from_numpy(a).to(dev)

    # resident panel + per-batch inputs
    if "phase" in stages:
        from eimp_b200.engine import Phaser
        Phaser(ctx, hm, sm, cm)   # uploads the typed reference used by the phasing kernels
    d_full = todev(panel.sitemajor)
    d_af = todev(panel.af.astype(np.float32))
    d_typed = todev(tg.typed.astype(np.int64))
    d_sitetyped = todev(sm)
    d_gt = todev(np.ascontiguousarray(tg.gt, dtype=np.uint8))
    phased_h = pack_rows(tg.truth, W(M))
    d_phased = todev(phased_h)
    ldb = (Mref + 63) // 64
    wM = W(M)
    do_phase = "phase" in stages
    from eimp_b200.engine import PhaseParams
    pparams = PhaseParams(K=cfg.K, beamwidth=cfg.beam).c()
    d_ph3 = torch.empty((nt, 2, wM), dtype=torch.int64, device=dev)     # phased haps, mat/pat interleaved
    d_mats = torch.empty((nt, wM), dtype=torch.int64, device=dev)
    d_pats = torch.empty((nt, wM), dtype=torch.int64, device=dev)
    d_pdm = torch.empty((nt, M), dtype=torch.float32, device=dev)
    d_pdp = torch.empty((nt, M), dtype=torch.float32, device=dev)
    d_tc = torch.empty(nt, dtype=torch.float32, device=dev)
    d_nc = torch.empty(nt, dtype=torch.int32, device=dev)
    d_dos = torch.empty((2 * nt, Mref), dtype=torch.float32, device=dev)
    d_bits = torch.empty((2 * nt, ldb), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    kern = {"phase": [], "smm": [], "dosage": []}

    def step_body():
        # the batch step without timing events (the CUDA-graph form captures this)
        ctx.check(L.eimp_imp_set_reference_dev(h, Mref, nh_ref, d_full.data_ptr(), d_af.data_ptr(), M,
                                               d_typed.data_ptr(), d_sitetyped.data_ptr()))
        if do_phase:
            ctx.check(L.eimp_phase_targets_dev(h, C.byref(pparams), nt, d_gt.data_ptr(), d_mats.data_ptr(),
                                               d_pats.data_ptr(), d_pdm.data_ptr(), d_pdp.data_ptr(),
                                               d_tc.data_ptr(), d_nc.data_ptr()))
            with torch.cuda.stream(stream):
                d_ph3[:, 0].copy_(d_mats)
                d_ph3[:, 1].copy_(d_pats)
        src = d_ph3 if do_phase else d_phased
        ctx.check(L.eimp_imp_prepare_dev(h, nt, src.data_ptr(), d_gt.data_ptr(), 0, 0, 0))
        ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, d_bits.data_ptr(), ldb, d_dos.data_ptr(), Mref))

    def step_timed():
        e = [ev() for _ in range(5)]
        e[0].record(stream)
        # the imputation reference (transposed panel, reference PBWT) depends on
        # the panel only: the library builds it on its side stream, overlapped
        # with the phasing below; the imputation calls wait for it
        ctx.check(L.eimp_imp_set_reference_dev(h, Mref, nh_ref, d_full.data_ptr(), d_af.data_ptr(), M,
                                               d_typed.data_ptr(), d_sitetyped.data_ptr()))
        if do_phase:
            ctx.check(L.eimp_phase_targets_dev(h, C.byref(pparams), nt, d_gt.data_ptr(), d_mats.data_ptr(),
                                               d_pats.data_ptr(), d_pdm.data_ptr(), d_pdp.data_ptr(),
                                               d_tc.data_ptr(), d_nc.data_ptr()))
            with torch.cuda.stream(stream):
                d_ph3[:, 0].copy_(d_mats)
                d_ph3[:, 1].copy_(d_pats)
            src = d_ph3
        else:
            src = d_phased
        e[1].record(stream)
        e[2].record(stream)
        ctx.check(L.eimp_imp_prepare_dev(h, nt, src.data_ptr(), d_gt.data_ptr(), 0, 0, 0))
        e[3].record(stream)
        ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, d_bits.data_ptr(), ldb, d_dos.data_ptr(), Mref))
        e[4].record(stream)
        return e

    def step_imp():
        step_timed()

    # beam-kernel roofline inputs: the library times its phasing stages with
    # CUDA events on its stream; the condensed rows of the batch (sum of 2S+1
    # over the targets) give the PBWT bytes the beam reads
    STAGES = ("prep", "split_readback", "cref", "pbwt", "beam")
    rows_total = 0
    if do_phase:
        ctx.check(L.eimp_set_timing(h, 1))
        rows_c = C.c_size_t(0)
        gt_host = np.ascontiguousarray(tg.gt, dtype=np.uint8)
        ctx.check(L.eimp_phase_cref_pbwt(h, C.byref(pparams), nt, gt_host.ctypes.data, C.byref(rows_c),
                                         None, None, None, None))
        rows_total = rows_c.value
    stage_ms = {k: [] for k in STAGES}

    for _ in range(args.warmup):
        step_imp()
    ctx.synchronize()
    # status check once (capacity errors would surface here)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ctx.launches
    evs = []
    st5 = (C.c_float * 5)()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        evs.append(step_timed())
        if do_phase:   # read before the next step's phasing records over them
            ctx.check(L.eimp_phase_stage_ms(h, st5, 5))
            for k, v in zip(STAGES, st5):
                stage_ms[k].append(float(v))
    ctx.synchronize()
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    clocks = sampler.stop()
    # the last timed step's outputs for the CPU sample's targets (compared with
    # the reference's own outputs once the CPU baseline has run)
    npar = min(args.cpu_sample_targets, nt)
    gpu_out = {"bits": d_bits[:2 * npar].cpu().numpy().view(np.uint64),
               "dos": d_dos[:2 * npar].cpu().numpy()}
    if do_phase:
        gpu_out.update(mats=d_mats[:npar].cpu().numpy().view(np.uint64),
                       pats=d_pats[:npar].cpu().numpy().view(np.uint64),
                       dm=d_pdm[:npar].cpu().numpy(), dp=d_pdp[:npar].cpu().numpy())
    step_ms = [e[0].elapsed_time(e[4]) for e in evs]
    for e in evs:
        kern["phase"].append(e[0].elapsed_time(e[1]))
        kern["smm"].append(e[2].elapsed_time(e[3]))   # includes any wait for the reference build
        kern["dosage"].append(e[3].elapsed_time(e[4]))
    tot_ms = float(np.sum(step_ms))
    if world > 1:
        t = torch.tensor([tot_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
        dist.barrier()
    dos_per_step = imputed_count(tg, Mref)
    value = world * dos_per_step * args.steps / (tot_ms / 1e3)

    # roofline of the dominant kernel.  With phasing that is the beam kernel
    # (more than half of the device time): its algorithmic bytes per launch are
    # one read of every target's condensed PBWT in both directions (2 x rows x
    # 2*ceil(K/32) uint32) plus the rows' zero counts, the genotype bytes it
    # reads and the phased haplotypes and dosages it writes.  Without phasing
    # it is the dosage kernel: dosage + bit outputs of every (haplotype, site)
    # + one read of the haplotype-major panel.
    peak, peak_kind = measured_peak_hbm()
    dos_ms = float(np.mean(kern["dosage"]))
    bytes_dos = 2 * nt * Mref * 4 + 2 * nt * ldb * 8 + nh_ref * W(Mref) * 8
    stage_means = {k: float(np.mean(v)) for k, v in kern.items()}
    if do_phase:
        stage_means.update({"phase_" + k: float(np.mean(v)) for k, v in stage_ms.items()})
        kw = 2 * ((min(cfg.K, nh_ref) + 31) // 32)
        beam_ms = float(np.mean(stage_ms["beam"]))
        bytes_beam = 2 * rows_total * kw * 4 + rows_total * 4 + nt * (M + 2 * W(M) * 8 + 2 * M * 4)
        achieved = bytes_beam / (beam_ms / 1e3) / 1e9
        # DRAM bytes of one beam launch: an ncu capture of the 64-target cfg2
        # launch (158.3 MB read + 13.1 MB written), scaled to the batch by
        # the number of targets
        traffic = (171.3e6 / 64) * nt if args.config == "cfg2" else None
        roofline = {"kernel": "beam_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                    "algorithmic_bytes_per_launch": bytes_beam, "avg_launch_ms": beam_ms,
                    "note": "latency-bound: one warp per target walks the beam sequentially",
                    "stage_ms": stage_means,
                    "dosage_kernel": {"achieved": bytes_dos / (dos_ms / 1e3) / 1e9, "avg_launch_ms": dos_ms,
                                      "algorithmic_bytes_per_launch": bytes_dos}}
    else:
        achieved = bytes_dos / (dos_ms / 1e3) / 1e9
        roofline = {"kernel": "dosage_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                    "algorithmic_bytes_per_launch": bytes_dos, "avg_launch_ms": dos_ms, "stage_ms": stage_means}

    # output statistics of the step's imputed bunch (the numbers of
    # VCFData::writeVCFImputedBunch: allele dosages and alleles written, r2,
    # AF, MAF, AC, AN, filters), timed on their own after the step: reads the
    # dosages and alleles of every (haplotype, site), writes the allele
    # dosages and alleles, 30 B per site of per-site inputs and outputs
    if do_phase:
        from eimp_b200._lib import EimpSiteStatsOpts
        d_ads = torch.empty_like(d_dos)
        d_gtb = torch.empty_like(d_bits)
        d_site = torch.empty(Mref * 6, dtype=torch.int32, device=dev)
        d_conf = torch.zeros(1, dtype=torch.int64, device=dev)
        so = EimpSiteStatsOpts(0, 0, 0.0, 0.0)
        sp = d_site.data_ptr()

        def stats_call():
            ctx.check(L.eimp_imp_site_stats_dev(h, 0, Mref, d_bits.data_ptr(), ldb, d_dos.data_ptr(), Mref,
                                                d_pdm.data_ptr(), d_pdp.data_ptr(), M, C.byref(so),
                                                d_ads.data_ptr(), Mref, d_gtb.data_ptr(), ldb, None, None, sp,
                                                sp + 4 * Mref, sp + 8 * Mref, sp + 12 * Mref, sp + 16 * Mref,
                                                sp + 20 * Mref, d_conf.data_ptr()))
        for _ in range(3):
            stats_call()
        st_ms = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = ev(), ev()
            e0.record(stream)
            stats_call()
            e1.record(stream)
            ctx.synchronize()
            st_ms.append(e0.elapsed_time(e1))
        st_ms = float(np.mean(st_ms))
        bytes_st = 2 * (2 * nt * Mref * 4 + 2 * nt * ldb * 8) + Mref * 30
        roofline["site_stats_kernel"] = {"achieved": bytes_st / (st_ms / 1e3) / 1e9, "avg_launch_ms": st_ms,
                                         "algorithmic_bytes_per_launch": bytes_st,
                                         "frac": bytes_st / (st_ms / 1e3) / 1e9 / peak}
        del d_ads, d_gtb

    # end to end through the public API: host (pinned) targets in, host dosages out
    e2e = None
    if rank == 0 or world > 1:
        ph_pin = torch.from_numpy(np.ascontiguousarray(phased_h).view(np.int64)).pin_memory()
        gt_pin = torch.from_numpy(np.ascontiguousarray(tg.gt, dtype=np.uint8)).pin_memory()
        dos_pin = torch.empty((2 * nt, Mref), dtype=torch.float32).pin_memory()
        bits_pin = torch.empty((2 * nt, W(Mref)), dtype=torch.int64).pin_memory()
        h2d = ph_pin.numel() * 8 + gt_pin.numel()
        d2h = dos_pin.numel() * 4 + bits_pin.numel() * 8

        mats_pin = torch.empty((nt, wM), dtype=torch.int64).pin_memory()
        pats_pin = torch.empty((nt, wM), dtype=torch.int64).pin_memory()
        pdm_pin = torch.empty((nt, M), dtype=torch.float32).pin_memory()
        pdp_pin = torch.empty((nt, M), dtype=torch.float32).pin_memory()
        tc_pin = torch.empty(nt, dtype=torch.float32).pin_memory()
        nc_pin = torch.empty(nt, dtype=torch.int32).pin_memory()
        if do_phase:
            h2d = 2 * gt_pin.numel() + ph_pin.numel() * 8   # genotypes (phasing + imputation) and phased haplotypes
            d2h += (mats_pin.numel() + pats_pin.numel()) * 8 + (pdm_pin.numel() + pdp_pin.numel()) * 4 + nt * 8

        def e2e_step():
            ctx.check(L.eimp_imp_set_reference_dev(h, Mref, nh_ref, d_full.data_ptr(), d_af.data_ptr(), M,
                                                   d_typed.data_ptr(), d_sitetyped.data_ptr()))
            if do_phase:
                # phasing through the host API (genotypes in, phased haplotypes and dosages out)
                ctx.check(L.eimp_phase_targets(h, C.byref(pparams), nt, gt_pin.data_ptr(), mats_pin.data_ptr(),
                                               pats_pin.data_ptr(), pdm_pin.data_ptr(), pdp_pin.data_ptr(),
                                               tc_pin.data_ptr(), nc_pin.data_ptr()))
                phv = ph_pin.view(nt, 2, wM)
                phv[:, 0].copy_(mats_pin)
                phv[:, 1].copy_(pats_pin)
            ctx.check(L.eimp_imp_prepare(h, nt, ph_pin.data_ptr(), gt_pin.data_ptr(), 0, 0, 0))
            ctx.check(L.eimp_imp_bunch(h, 0, Mref, bits_pin.data_ptr(), dos_pin.data_ptr()))
        e2e_step()
        ctx.synchronize()
        t0 = time.perf_counter()
        n_e2e = max(1, min(args.steps, 3))
        for _ in range(n_e2e):
            e2e_step()
        ctx.synchronize()
        dt = (time.perf_counter() - t0) / n_e2e
        e2e = {"value": world * dos_per_step / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3}

    # the CUDA-graph form: the same step captured once (phasing in capacity
    # mode, the rows reserved for this batch) and replayed; its outputs must
    # equal the eager step's
    graph = None
    if args.graph_steps > 0 and do_phase:
        ref_out = [d_dos.clone(), d_bits.clone(), d_mats.clone(), d_pats.clone()]
        ctx.check(L.eimp_set_timing(h, 0))
        ctx.check(L.eimp_phase_reserve(h, C.byref(pparams), nt, rows_total))
        step_body()
        ctx.synchronize()
        ctx.check(L.eimp_capture_begin(h))
        step_body()
        ctx.check(L.eimp_capture_end(h))
        for _ in range(args.warmup):
            ctx.check(L.eimp_graph_launch(h))
        ctx.synchronize()
        gms = []
        for _ in range(args.graph_steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            g0, g1 = ev(), ev()
            g0.record(stream)
            ctx.check(L.eimp_graph_launch(h))
            g1.record(stream)
            gms.append((g0, g1))
        ctx.synchronize()
        torch.cuda.synchronize()
        g_ms = float(np.mean([a.elapsed_time(b) for a, b in gms]))
        same = all(torch.equal(a, b) for a, b in zip(ref_out, [d_dos, d_bits, d_mats, d_pats]))
        graph = {"value": world * dos_per_step / (g_ms / 1e3), "unit": UNIT, "ms_per_step": g_ms,
                 "steps": args.graph_steps, "equal_to_eager": bool(same), "rows_reserved": int(rows_total)}
        ctx.check(L.eimp_phase_reserve(h, C.byref(pparams), nt, 0))
        ctx.check(L.eimp_set_timing(h, 1))

    # the panel's Qref haplotype section (qref_spec.md section I) decoded on
    # the device into the site-major rows: the section already in HBM (value),
    # and through the host API from host memory (index walk, one copy,
    # decode); the reference's own decoder on one host core beside it
    qref = None
    if args.qref_steps > 0 and rank == 0:
        sec = synth.qref_section(panel.sitemajor)
        nwq = W(nh_ref)
        offs = np.zeros(Mref, np.int64)
        assert L.eimp_qref_index(sec.ctypes.data, sec.size, Mref, nh_ref // 2, offs.ctypes.data) == 0
        d_sec = torch.zeros(sec.size + 16, dtype=torch.uint8, device=dev)
        d_sec[:sec.size].copy_(torch.from_numpy(sec))
        d_offs = torch.from_numpy(offs).to(dev)
        d_rows = torch.empty(Mref * nwq, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()

        def qcall():
            ctx.check(L.eimp_qref_decode_dev(h, d_sec.data_ptr(), d_offs.data_ptr(), Mref, nh_ref // 2,
                                             d_rows.data_ptr(), nwq))
        for _ in range(3):
            qcall()
        ctx.synchronize()
        qms = []
        for _ in range(args.qref_steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            q0, q1 = ev(), ev()
            q0.record(stream)
            qcall()
            q1.record(stream)
            ctx.synchronize()
            qms.append(q0.elapsed_time(q1))
        q_ms = float(np.mean(qms))
        same = torch.equal(d_rows.view(Mref, nwq), d_full.view(Mref, -1))
        sec_pin = torch.from_numpy(sec).pin_memory()
        ctx.check(L.eimp_qref_decode(h, sec_pin.data_ptr(), sec.size, Mref, nh_ref // 2, d_rows.data_ptr(), nwq,
                                     None))   # the context's staging buffers reach their size
        t0 = time.perf_counter()
        ctx.check(L.eimp_qref_decode(h, sec_pin.data_ptr(), sec.size, Mref, nh_ref // 2, d_rows.data_ptr(), nwq,
                                     None))
        e2e_ms = (time.perf_counter() - t0) * 1e3
        qbytes = sec.size + Mref * nwq * 8
        qref = {"variants": Mref, "haplotypes": nh_ref, "section_bytes": int(sec.size),
                "coded_variants": int(sum(1 for o in offs if int(sec[o:o + 8].view(np.uint64)[0]) > 0)),
                "value": Mref / (q_ms / 1e3), "unit": "variants/s", "ms": q_ms,
                "roofline": {"bound": "hbm", "achieved": qbytes / (q_ms / 1e3) / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": qbytes / (q_ms / 1e3) / 1e9 / peak,
                             "algorithmic_bytes_per_launch": qbytes},
                "e2e": {"value": Mref / (e2e_ms / 1e3), "unit": "variants/s", "ms": e2e_ms,
                        "h2d_bytes": int(sec.size), "d2h_bytes": 0},
                "equal_to_panel": bool(same)}
        if not args.no_cpu_baseline:
            from oracle import refcore
            if refcore.available():
                t0 = time.perf_counter()
                _, rc = refcore.qref_decode(sec, Mref, nwq)
                c_s = time.perf_counter() - t0
                qref["cpu_baseline"] = {"value": Mref / c_s, "unit": "variants/s", "cores": 1, "kind": "reference",
                                        "sample": f"all {Mref} variants, runlengthDecode of utils.h", "ok": rc == 0}
        del d_sec, d_rows, d_offs

    # the plain drop-in form: one target per call (phase, matches, dosages),
    # device-resident inputs, on a sample of targets; same metric
    plain = None
    if rank == 0 and args.plain_targets > 0:
        npl = min(args.plain_targets, nt)
        ep = [ev() for _ in range(2)]
        torch.cuda.synchronize()
        ep[0].record(stream)
        for i in range(npl):
            if do_phase:
                ctx.check(L.eimp_phase_targets_dev(h, C.byref(pparams), 1, d_gt[i:i + 1].data_ptr(),
                                                   d_mats[i:i + 1].data_ptr(), d_pats[i:i + 1].data_ptr(),
                                                   d_pdm[i:i + 1].data_ptr(), d_pdp[i:i + 1].data_ptr(),
                                                   d_tc[i:i + 1].data_ptr(), d_nc[i:i + 1].data_ptr()))
                with torch.cuda.stream(stream):
                    d_ph3[i, 0].copy_(d_mats[i])
                    d_ph3[i, 1].copy_(d_pats[i])
                src1 = d_ph3[i]
            else:
                src1 = d_phased[2 * i:2 * i + 2]
            ctx.check(L.eimp_imp_prepare_dev(h, 1, src1.data_ptr(), d_gt[i:i + 1].data_ptr(), 0, 0, 0))
            ctx.check(L.eimp_imp_bunch_dev(h, 0, Mref, d_bits[2 * i:2 * i + 2].data_ptr(), ldb,
                                           d_dos[2 * i:2 * i + 2].data_ptr(), Mref))
        ep[1].record(stream)
        ctx.synchronize()
        pl_ms = ep[0].elapsed_time(ep[1])
        sub = synth.Targets(tg.typed, tg.gt[:npl], tg.truth[:2 * npl])
        pl_value = imputed_count(sub, Mref) / (pl_ms / 1e3)
        plain = {"value": pl_value, "unit": UNIT, "targets": npl, "ms_per_target": pl_ms / npl,
                 "batched_over_plain": (value / world) / pl_value,
                 "form": "one target per call: eimp_phase_targets_dev, eimp_imp_prepare_dev, eimp_imp_bunch_dev"}

    # serving: continuous batching of requests of 1..256 targets arriving as a
    # Poisson stream, two slots (contexts) on this device; host buffers in
    # and out; latency from submission to result
    serving = None
    if rank == 0 and args.serving_requests > 0 and do_phase:
        from eimp_b200.engine import PhaseParams as PP
        from eimp_b200.serving import GpuSlot, Server, device_bytes_per_target, load_test
        srng = np.random.default_rng(cfg.seed + 7)
        sizes = np.exp(srng.uniform(0.0, np.log(256.0), size=args.serving_requests)).astype(int).clip(1, 256)
        reqs, o = [], 0
        for sz in sizes:
            idx = (o + np.arange(sz)) % nt
            reqs.append(np.ascontiguousarray(tg.gt[idx]))
            o += sz
        pp = PP(K=cfg.K, beamwidth=cfg.beam)
        slots = [GpuSlot(local, hm, sm, cm, panel.sitemajor, panel.af.astype(np.float32), tg.typed, nh_ref, pp)
                 for _ in range(2)]
        bpt = device_bytes_per_target(M, Mref, min(cfg.K, nh_ref), P=cfg.beam)
        free_b, _tot = torch.cuda.mem_get_info(dev)
        srv = Server(slots, max_batch_targets=512, mem_budget=0.5 * free_b, bytes_per_target=bpt)
        srv.warmup(tg.gt[np.arange(512) % nt])   # buffers at their working size
        rate = args.serving_rate
        cnt = lambda g: int(2 * ((Mref - M) * g.shape[0] + (g == 3).sum()))  # noqa: E731
        serving = load_test(srv, reqs, rate, seed=cfg.seed, count=cnt)
        srv.close()
        serving.update({"unit": UNIT, "slots": 2, "max_batch_targets": 512,
                        "request_sizes": "log-uniform 1..256 targets", "arrivals": "Poisson"})

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        ref_out = {}
        cpu, _ = cpu_baseline(cfg, panel, tg, npar, stages, keep=ref_out)
        if ref_out:
            parity = parity_block(gpu_out, ref_out, cfg, panel, tg, npar, stages)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64/f32",
                "data": "synthetic (seeded Li-Stephens mosaics of the configuration's shape)",
                "config": config_block(cfg, panel, tg, stages), "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "clocks": clocks, "gpu_launches": int(launches), "plain": plain, "serving": serving,
                "graph": graph, "qref_decode": qref, "parity": parity}
        if do_phase:
            line["phased_samples_per_sec"] = world * nt * args.steps / (tot_ms / 1e3)
            line["phase_ms_per_step"] = float(np.mean(kern["phase"]))
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
