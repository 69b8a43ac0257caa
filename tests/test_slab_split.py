"""The y-slab split's host side on the CPU (lbl/slab.py): the band partition, the halo row
plan that lbl_slab_pack / lbl_slab_unpack implement, and the ring exchange over gloo ranks.

The ranks' compute here is the FP64 oracle (oracle/oracle.cpp): each rank advances its band
(own rows plus halos, as a periodic grid) with the oracle's step and analysis, exchanges
halos through `ring_exchange` by the row plan, and must reproduce the whole-grid oracle run
on its own rows bit for bit.  Two things the engine does in the library are done here by
hand: the band's constants are the whole grid's (an h_ref giving the same dx) and its force
field is the whole grid's rows.  The oracle's set_f takes FP32, so both runs round their
state to FP32 after every step and analysis in the same way."""
import datetime
import math
import multiprocessing
import os
import socket

import numpy as np
import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")

NX, M, STEPS_A, STEPS_B = 64, 4, 6, 5


def test_partition_covers_the_grid_in_aligned_bands():
    from lbl import slab
    for ny, world, align in [(256, 1, 8), (256, 2, 8), (256, 3, 8), (64, 4, 8), (100, 3, 1), (96, 5, 4)]:
        bands = slab.partition(ny, world, align)
        assert bands[0][0] == 0 and sum(o for _, o in bands) == ny
        assert all(b[0] + b[1] == c[0] for b, c in zip(bands, bands[1:]))
        assert all(r0 % align == 0 and o % align == 0 for r0, o in bands)
        assert max(o for _, o in bands) - min(o for _, o in bands) <= align
    with pytest.raises(ValueError):
        slab.partition(100, 2, 8)
    with pytest.raises(ValueError):
        slab.partition(64, 9, 8)


def test_halo_plan_and_reach():
    import lbl
    from lbl import slab
    plan = slab.halo_rows(48, 8, 4)
    assert plan == {"to_prev": (12, 16), "to_next": (32, 36), "from_prev": (0, 4), "from_next": (44, 48)}
    with pytest.raises(ValueError):
        slab.halo_rows(48, 8, 9)
    c1 = lbl.config_default("DA_LETKF", 256, 16, da_xyprune=4, letkf_rloc_len=1)
    assert slab.window_reach(c1) == 8 and slab.default_halo(c1) == 8 and slab.row_align(c1) == 8
    assert slab.window_reach(lbl.config_default("DA_LETKF", 256, 16, da_xyprune=4, letkf_rloc_len=0)) == 8
    assert slab.default_halo(lbl.config_default("DA_LETKF", 96, 4, da_xyprune=3, letkf_rloc_len=2)) == 24
    assert slab.default_halo(lbl.config_default("NATURE", 256, 16)) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _band_h_ref(h_ref, ny_global, ny_local):
    """An h_ref for which the band's dx = float(h_ref) / float(ny_local - 1) is the whole grid's."""
    dx = np.float32(np.float32(h_ref) / np.float32(ny_global - 1))
    x0 = np.float32(dx * np.float32(ny_local - 1))
    for toward in (np.float32(np.inf), np.float32(-np.inf)):
        x = x0
        for _ in range(16):
            if np.float32(x / np.float32(ny_local - 1)) == dx:
                return float(x)
            x = np.nextafter(x, toward)
    raise AssertionError("no h_ref reproduces the grid's dx")


def _worker(rank, world, port, mode, halo, bands, out):
    import sys
    sys.path.insert(0, ROOT)
    for p in ("lbm2d-letkf_b200", "oracle"):
        sys.path.insert(0, os.path.join(ROOT, p))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    import oracle
    from lbl import slab
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        oracle.set_threads(1)
        ny = NX
        gcfg = oracle.config_default(mode, NX, M, da_xyprune=4, letkf_rloc_len=1, obs_error_u=0.1,
                                     obs_error_rho=0.01)
        assert halo >= slab.default_halo(gcfg)
        row0, own = bands[rank]
        nyl = own + 2 * halo
        rows = (row0 - halo + np.arange(nyl)) % ny
        bcfg = gcfg.copy()
        bcfg.ny = nyl
        bcfg.h_ref = _band_h_ref(gcfg.h_ref, ny, nyl)
        g, b = oracle.Oracle(gcfg), oracle.Oracle(bcfg)
        g.init(0)
        rng = np.random.default_rng(7)
        kx, _, _ = oracle.force_modes(gcfg)
        fx, fy = g.force(rng.normal(0, 0.84, 4 * len(kx)).astype(np.float32))
        fx, fy = fx.astype(np.float32), fy.astype(np.float32)
        g.set_force(fx, fy)
        b.set_force(fx[rows], fy[rows])
        for m in range(M):
            fm = g.get_f(m).astype(np.float32)
            g.set_f(m, fm)
            b.set_f(m, fm[:, rows])
        group = dist.group.WORLD
        nb = M * 9 * halo * NX
        bufs = {k: torch.zeros(nb, dtype=torch.float64) for k in ("send_prev", "send_next", "recv_prev", "recv_next")}

        def exchange(k):
            plan = slab.halo_rows(nyl, halo, k)
            f = np.stack([b.get_f(m) for m in range(M)])  # (M, 9, nyl, NX) FP64
            n = M * 9 * k * NX
            bufs["send_prev"][:n] = torch.from_numpy(f[:, :, slice(*plan["to_prev"])].ravel())
            bufs["send_next"][:n] = torch.from_numpy(f[:, :, slice(*plan["to_next"])].ravel())
            slab.ring_exchange(group, bufs["send_prev"][:n], bufs["send_next"][:n], bufs["recv_prev"][:n],
                               bufs["recv_next"][:n])
            f[:, :, slice(*plan["from_prev"])] = bufs["recv_prev"][:n].numpy().reshape(M, 9, k, NX)
            f[:, :, slice(*plan["from_next"])] = bufs["recv_next"][:n].numpy().reshape(M, 9, k, NX)
            for m in range(M):
                b.set_f(m, f[m].astype(np.float32))

        def steps(n):
            # at most halo / 2 steps between exchanges; both runs round to FP32 after each step
            left = n
            while left:
                k = min(halo // 2, left)
                for _ in range(k):
                    g.step_noforce()
                    b.step_noforce()
                    for m in range(M):
                        g.set_f(m, g.get_f(m).astype(np.float32))
                        b.set_f(m, b.get_f(m).astype(np.float32))
                exchange(2 * k)
                left -= k

        steps(STEPS_A)
        if mode == "DA_LETKF":
            r, u, v = g.macros(0)
            noise = np.random.default_rng(11)
            ro = (r + noise.normal(0, 0.01, r.shape)).astype(np.float32)
            uo = (u + noise.normal(0, 0.1, u.shape) * 0.01).astype(np.float32)
            vo = (v + noise.normal(0, 0.1, v.shape) * 0.01).astype(np.float32)
            g.assimilate(ro, uo, vo)
            b.assimilate(ro[rows], uo[rows], vo[rows])
            for m in range(M):  # the band's state is rounded in the exchange
                g.set_f(m, g.get_f(m).astype(np.float32))
            exchange(halo)
            steps(STEPS_B)
        worst = 0.0
        for m in range(M):
            want = g.get_f(m)[:, row0:row0 + own]
            got = b.get_f(m)[:, halo:halo + own]
            worst = max(worst, float(np.abs(got - want).max()))
        out.put((rank, worst, row0, own))
    finally:
        dist.destroy_process_group()


# (the band heights avoid those own + 2 halo for which no FP32 h_ref gives the grid's dx)
@pytest.mark.parametrize("mode,halo,bands", [
    ("NATURE", 2, [(0, 32), (32, 32)]),                  # one step per exchange
    ("NATURE", 4, [(0, 20), (20, 20), (40, 24)]),        # uneven bands, two steps per exchange
    ("DA_LETKF", 8, [(0, 32), (32, 32)]),                # C1's window reach and alignment
    ("DA_LETKF", 8, [(0, 24), (24, 24), (48, 16)]),
])
def test_bands_reproduce_the_whole_grid_over_gloo(mode, halo, bands):
    world = len(bands)
    ctx = multiprocessing.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, halo, bands, out)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted(out.get(timeout=240) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert sum(own for _, _, _, own in res) == NX
    for rank, worst, row0, own in res:
        assert worst == 0.0, (rank, worst)
