"""The batched form (eimp_b200/batch.py): several array densities over one
resident panel, each density group on its own context and streams with its
targets phased in capacity-mode batches, all groups enqueued at once and
overlapping on the device.  Every group's phased haplotypes, phasing
dosages, imputed alleles and dosages must equal the plain per-group calls
(Phaser / PBWTImputer, themselves bit-exact against the reference), and the
CUDA-graph replay of the step must equal the eager step."""
import numpy as np
import pytest

from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def test_density_groups_concurrent_and_graph(ctx):
    import torch
    from eimp_b200 import synth
    from eimp_b200.batch import DensityGroup, enqueue_step
    from eimp_b200.engine import PBWTImputer, PhaseParams, Phaser
    panel, groups = synth.generate("cfg1")
    base = groups[0]
    rng = np.random.default_rng(3)
    # three typed-site sets of the cfg1 panel: 5 %, 10 % (the group as
    # generated) and 15 % of the sites, missingness U(0, 5 %)
    sets = []
    truth_all = base.truth
    for frac, nt in ((0.05, 9), (0.10, 14), (0.15, 7)):
        if frac == 0.10:
            sets.append((base.typed, base.gt[:nt]))
            continue
        typed = np.sort(rng.choice(panel.nsites, int(frac * panel.nsites), replace=False)).astype(np.int64)
        # genotypes at the new typed sites from panel haplotypes (mosaic-like targets)
        from eimp_b200.bits import gather_bits
        haps = panel.hapmajor[rng.integers(0, panel.nhaps, 2 * nt)]
        th = gather_bits(haps, typed)
        gt = (th[0::2] + th[1::2]).astype(np.uint8)
        gt[rng.random(gt.shape) < rng.uniform(0, 0.05, (nt, 1))] = 3
        sets.append((typed, gt))
    dev = torch.device("cuda", 0)
    d_full = torch.from_numpy(panel.sitemajor.view(np.int64)).to(dev)
    d_af = torch.from_numpy(panel.af.astype(np.float32)).to(dev)
    pp = PhaseParams(K=1024, beamwidth=64)
    grp = []
    for typed, gt in sets:
        hm, sm, cm = synth.typed_views(panel, typed)
        grp.append(DensityGroup(0, d_full, d_af, panel.nhaps, typed, hm, sm, cm, gt, pp, batch_targets=4))
    assert [len(g.batches) for g in grp] == [3, 4, 2]
    enqueue_step(grp)
    torch.cuda.synchronize()
    for g in grp:
        g.ctx.synchronize()
    eager = [(g.d_mats.clone(), g.d_pats.clone(), g.d_pdm.clone(), g.d_pdp.clone(), g.d_dos.clone(),
              g.d_bits.clone()) for g in grp]
    for (typed, gt), out in zip(sets, eager):
        hm, sm, cm = synth.typed_views(panel, typed)
        mats, pats, dm, dp, tc, nc = Phaser(ctx, hm, sm, cm).phase(pp, gt)
        np.testing.assert_array_equal(out[0].cpu().numpy().view(np.uint64), mats)
        np.testing.assert_array_equal(out[1].cpu().numpy().view(np.uint64), pats)
        np.testing.assert_array_equal(out[2].cpu().numpy(), dm)
        np.testing.assert_array_equal(out[3].cpu().numpy(), dp)
        ph = np.zeros((2 * gt.shape[0], W(len(typed))), np.uint64)
        ph[0::2], ph[1::2] = mats, pats
        imp = PBWTImputer(ctx, panel.sitemajor, panel.af, typed, sm, panel.nhaps)
        imp.prepareImputation(ph, gt)
        bits, dos = imp.impute_window(0, panel.nsites)
        np.testing.assert_array_equal(out[4].cpu().numpy(), dos)
        nb = (panel.nsites + 63) // 64
        np.testing.assert_array_equal(out[5].cpu().numpy().view(np.uint64), bits[:, :nb])
    # the graph form: one captured step per group, replayed concurrently
    for g in grp:
        g.d_dos.zero_()
        g.d_mats.zero_()
        g.capture()
    for _ in range(2):
        enqueue_step(grp, capture_graphs=True)
    torch.cuda.synchronize()
    for g, out in zip(grp, eager):
        g.ctx.synchronize()
        assert torch.equal(g.d_mats, out[0]) and torch.equal(g.d_dos, out[4]) and torch.equal(g.d_bits, out[5])
    for g in grp:
        g.close()
