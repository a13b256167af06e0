"""Launch-shape autotuner for the batched form.

The kernels' results do not depend on their launch shapes, only their speed
does, and the best shape depends on the workload: how many target haplotypes
and sites the dosage kernel covers, how large the match trees grow, how many
targets a beam launch gets and how unevenly long they are.  The tuner times
every candidate of each knob on a density group's own data (the other knobs
at their current values), keeps the fastest and leaves it set on the group's
context.  Knobs (eimp_set_launch_shape, include/eimp_gpu.h):

  dosage_span     64-site tiles per warp of the dosage kernel       4, 8, 16
  smm_warps       target haplotypes per CTA of the match search     1, 2, 4
  beam_slots_pct  warps of the persistent beam, % of the resident   100, 75, 50
  smm_tree_pools  large match trees go on in global pools (1) or    1, 0
                  are redone by the retry launch (0)

Timing is on the device (CUDA events on the group's stream), best of
``reps`` runs; the phasing knob is timed over all of the group's batches.

Alone, every group wants all of the SMs for its beam.  In a step the groups
run side by side and the densest group's chain of kernels is the critical
path, so :func:`tune_step_shares` then times whole steps with the lighter
groups' beams held to smaller shares of the resident warps (their kernels
still overlap the dense group's) and keeps the fastest.
"""
from __future__ import annotations

import ctypes as C

KNOBS = {
    "dosage_span": (0, (4, 8, 16)),
    "smm_warps": (1, (1, 2, 4)),
    "beam_slots_pct": (2, (100, 75, 50)),
    "smm_tree_pools": (3, (1, 0)),
}


def get(group, knob: str) -> int:
    v = C.c_int(0)
    group.ctx.check(group.L.eimp_get_launch_shape(group.h, KNOBS[knob][0], C.byref(v)))
    return int(v.value)


def set_shape(group, knob: str, value: int):
    group.ctx.check(group.L.eimp_set_launch_shape(group.h, KNOBS[knob][0], int(value)))


def _time(group, fn, reps: int) -> float:
    import torch
    best = float("inf")
    for _ in range(reps):
        group.ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(group.stream)
        fn()
        e1.record(group.stream)
        group.ctx.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune_group(group, reps: int = 2,
               knobs=("dosage_span", "smm_warps", "smm_tree_pools", "beam_slots_pct")) -> dict:
    """Tunes the knobs of one DensityGroup (eimp_b200/batch.py) on its data;
    returns {knob: {"chosen": value, "ms": {value: best ms}}}."""
    group.enqueue()   # a full step first: the phased haplotypes and the reference exist
    group.ctx.synchronize()
    stage = {
        "dosage_span": lambda: group.L.eimp_imp_bunch_dev(group.h, 0, group.Mref, group.d_bits.data_ptr(), group.ldb,
                                                          group.d_dos.data_ptr(), group.Mref),
        "smm_warps": lambda: group.L.eimp_imp_prepare_dev(group.h, group.nt, group.d_ph.data_ptr(),
                                                          group.d_gt.data_ptr(), 0, 0, 0),
        "smm_tree_pools": lambda: group.L.eimp_imp_prepare_dev(group.h, group.nt, group.d_ph.data_ptr(),
                                                               group.d_gt.data_ptr(), 0, 0, 0),
        "beam_slots_pct": group.phase,
    }
    out = {}
    for k in knobs:
        times = {}
        for v in KNOBS[k][1]:
            set_shape(group, k, v)
            fn = stage[k]

            def run(fn=fn):
                rc = fn()
                if isinstance(rc, int) and rc:
                    group.ctx.check(rc)
            times[v] = _time(group, run, 1 if k.startswith("beam") else reps)
        best = min(times, key=times.get)
        set_shape(group, k, best)
        out[k] = {"chosen": best, "ms": {str(v): round(t, 3) for v, t in times.items()}}
    # the tuned step's outputs (the last candidate ran last)
    group.enqueue()
    group.ctx.synchronize()
    return out


def tune_step_shares(groups, reps: int = 1) -> dict:
    """Step-level choice of the beam shares: the groups with the most
    condensed rows keep their own choice, the lighter ones get each candidate
    share set in turn (uniform 100, 75 or 50 %, or graded from 50 % for the
    lightest up to 75 %); whole steps are timed on the device and the fastest
    set stays on the groups.  Returns {"chosen": [...], "ms": {label: ms}}."""
    import torch
    from .batch import enqueue_step, step_order
    order = step_order(groups)            # heaviest first
    light = order[1:]
    if not light:
        return {"chosen": [get(g, "beam_slots_pct") for g in groups], "ms": {}}
    graded = {i: (50 if r == len(light) - 1 else 75) for r, i in enumerate(light)}
    cands = {"own": {i: get(groups[i], "beam_slots_pct") for i in light},
             "75": {i: 75 for i in light}, "50": {i: 50 for i in light}, "graded": graded}
    dev = groups[0].dev
    main = torch.cuda.current_stream(dev)
    times = {}
    for label, shares in cands.items():
        for i, v in shares.items():
            set_shape(groups[i], "beam_slots_pct", v)
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            for e in enqueue_step(groups, e0):
                main.wait_event(e)
            e1.record(main)
            torch.cuda.synchronize(dev)
            for g in groups:
                g.ctx.synchronize()
            best = min(best, e0.elapsed_time(e1))
        times[label] = round(best, 3)
    label = min(times, key=times.get)
    for i, v in cands[label].items():
        set_shape(groups[i], "beam_slots_pct", v)
    return {"chosen": [get(g, "beam_slots_pct") for g in groups], "label": label, "ms": times}
