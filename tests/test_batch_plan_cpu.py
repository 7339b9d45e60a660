"""The cluster-resident batch kernel's plan (host logic, no GPU): lattices on
clusters, rows on CTAs, shared-memory layout and halo sources.  The kernel
indexes shared memory, and reads its peers' shared memory, only through this
plan, so every rule the kernel relies on is checked here:

* each lattice lives in one cluster, and each of its rows in exactly one
  segment of one CTA of that cluster;
* a CTA's segments are laid out back to back ([halo row, core rows, halo
  row] each), its sites numbered back to back;
* the halo rows above and below a segment come from the CTA and slot that
  hold rows r0 - 1 and r0 + rows (mod N) of the same lattice;
* the shared memory the plan asks for covers every CTA's layout;
* clusters are balanced longest-first, CTAs within one row of an even split.
"""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd


def check_plan(sizes, S, C):
    ctas, segs, smem, fits = asd.batch_plan_clusters(sizes, S, C, smem_limit=1 << 40)
    assert fits
    assert ctas.shape == (S * C, 4)
    owner = {}  # (lattice, row) -> (cluster, rank, slot)
    max_buf = max_sites = 0
    for b, (seg0, nseg, nsites, buf) in enumerate(ctas):
        c, rank = divmod(b, S)
        base = core = 0
        for k in range(seg0, seg0 + nseg):
            lat, N, r0, rows, sbase, core0 = segs[k][:6]
            assert N == sizes[lat] and rows >= 1 and 0 <= r0 and r0 + rows <= N
            assert sbase == base and core0 == core
            for r in range(rows):
                key = (lat, r0 + r)
                assert key not in owner, key
                owner[key] = (c, rank, sbase + (r + 1) * N)
            base += (rows + 2) * N
            core += rows * N
        assert nsites == core and buf == max(base, 1)
        max_buf, max_sites = max(max_buf, buf), max(max_sites, nsites)
    assert set(owner) == {(l, r) for l, n in enumerate(sizes) for r in range(n)}
    clusters_of = {}
    for (lat, _), (c, _, _) in owner.items():
        clusters_of.setdefault(lat, set()).add(c)
    assert all(len(v) == 1 for v in clusters_of.values())
    for b, (seg0, nseg, _, _) in enumerate(ctas):
        c = b // S
        for k in range(seg0, seg0 + nseg):
            lat, N, r0, rows = segs[k][:4]
            for (rank, off, rbuf), want in ((segs[k][6:9], (r0 - 1) % N),
                                            (segs[k][9:12], (r0 + rows) % N)):
                oc, orank, oslot = owner[(lat, want)]
                assert (oc, orank, oslot) == (c, rank, off)
                assert rbuf == ctas[c * S + rank][3]
    assert smem == 4 * (6 * max_buf + 6 * max_sites)
    # balance: clusters longest first; CTAs within one row of an even split
    load = np.zeros(C)
    for lat, (c,) in clusters_of.items():
        load[c] += sizes[lat] ** 2
    for c in range(C):
        per = ctas[c * S:(c + 1) * S, 2]
        widest = max([sizes[l] for l, cs in clusters_of.items() if c in cs], default=0)
        assert per.max() <= -(-load[c] // S) + widest
    return ctas, segs, smem


@pytest.mark.parametrize("sizes,S,C", [
    ([int(x) for x in np.random.default_rng(5).choice([48, 64, 96, 128, 160], size=48)], 6, 22),
    ([64] * 132, 1, 148),
    ([48, 64, 37, 96, 5, 128, 160, 20], 8, 18),   # 10 empty clusters
    ([3, 4, 5, 7, 11, 13, 160], 3, 4),
    ([160], 8, 1),                                 # one lattice over 8 CTAs
    ([5, 5, 5], 8, 2),                             # more CTAs than rows
    ([int(x) for x in np.random.default_rng(9).integers(3, 120, size=40)], 5, 7),
])
def test_cluster_plan(sizes, S, C):
    check_plan(sizes, S, C)


def test_cluster_plan_reports_what_does_not_fit():
    """One 160^2 lattice on single-CTA clusters: 1.2 MB of shared memory."""
    _, _, smem, fits = asd.batch_plan_clusters([160], 1, 1, smem_limit=232448)
    assert not fits and smem > 232448
    _, _, smem, fits = asd.batch_plan_clusters([160], 8, 1, smem_limit=232448)
    assert fits and smem <= 232448
