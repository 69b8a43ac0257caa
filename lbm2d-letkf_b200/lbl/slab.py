"""y-slab split of one DA experiment over ranks (lbl_slab_set, lbl_slab_pack, lbl_slab_unpack).

The reference spreads one experiment over MPI ranks by member: rank k advances member k,
and every analysis transposes the ensemble all-to-all so that each rank analyses a batch of
grid rows (src/util/letkf_solver.h:135-215, 374-394; src/letkf.cu:191, 273, 315).  Here
every rank holds ALL members of a band of rows instead, so the analysis needs no transpose and
the only traffic is a halo of rows between neighbouring bands:

* rank r owns the rows [row0, row0 + own) and keeps `halo` rows of each neighbour beside
  them; its context runs every kernel over the own + 2 halo rows as if they were periodic;
* k steps corrupt the outer 2k rows on each side, so after at most halo / 2 steps each
  rank sends 2k rows to each neighbour (one packed buffer of all members and directions per
  neighbour), and after an analysis all `halo` rows (the analysis of halo rows reads past the
  band);
* a forecast computes its forcing once (lbl_slab_forecast_begin) and advances in chunks of
  halo / 2 steps (lbl_slab_forecast_chunk), the exchange between chunks;
* the own rows then equal the single-context run bit for bit.

`ring_exchange` moves the packed buffers with torch.distributed point-to-point operations
(NCCL between GPUs, on the engine's stream; gloo on the CPU).  `SlabExperiment` drives
either one band per process (a process group) or every band of the experiment in this
process on one device, the neighbours' buffers read in place.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

import lbl

__all__ = ["partition", "window_reach", "default_halo", "halo_rows", "ring_exchange", "SlabExperiment"]


def window_reach(cfg) -> int:
    """Rows between a grid point and the farthest observation site of its LETKF window:
    n_obs_local * DA_XYPRUNE (letkf.cu:45-55), 0 outside DA_LETKF."""
    if cfg.mode != lbl.MODE_DA_LETKF:
        return 0
    p = cfg.da_xyprune
    nl = (0 if p == 1 else 2) if cfg.letkf_rloc_len <= 0 else 2 * cfg.letkf_rloc_len
    return nl * p


def row_align(cfg) -> int:
    """Band boundaries and halos fall on observation sites and analysis tiles under DA_LETKF."""
    if cfg.mode != lbl.MODE_DA_LETKF:
        return 1
    return 8 * cfg.da_xyprune // math.gcd(8, cfg.da_xyprune)


def default_halo(cfg) -> int:
    """The smallest valid halo: 2 rows for a forecast, the window reach (rounded up to the
    alignment) for DA_LETKF."""
    a = row_align(cfg)
    h = max(2, window_reach(cfg))
    return (h + a - 1) // a * a


def partition(ny: int, world: int, align: int = 1) -> List[Tuple[int, int]]:
    """(row0, own) of each rank: ny rows in `world` bands of whole multiples of `align`,
    the first ones one unit larger when they do not divide evenly."""
    if ny % align:
        raise ValueError(f"ny = {ny} is not a multiple of the band alignment {align}")
    units = ny // align
    if units < world:
        raise ValueError(f"{ny} rows do not make {world} bands of {align}-row units")
    base, extra = divmod(units, world)
    out, row0 = [], 0
    for r in range(world):
        own = (base + (r < extra)) * align
        out.append((row0, own))
        row0 += own
    return out


def halo_rows(ny_local: int, halo: int, rows: int) -> dict:
    """The local row ranges [a, b) of one exchange of `rows` rows (lbl_slab_pack /
    lbl_slab_unpack): sent to the previous and next band, received from them."""
    if not 1 <= rows <= halo:
        raise ValueError("rows must lie in [1, halo]")
    return {"to_prev": (2 * halo - rows, 2 * halo), "to_next": (ny_local - 2 * halo, ny_local - 2 * halo + rows),
            "from_prev": (0, rows), "from_next": (ny_local - rows, ny_local)}


def ring_exchange(group, send_prev, send_next, recv_prev, recv_next):
    """Send send_prev to the previous rank and send_next to the next one, receiving the
    previous rank's send_next into recv_prev and the next rank's send_prev into recv_next
    (ranks in a ring).  The four transfers are posted together; with NCCL they run after
    the current stream's work and the current stream waits for them."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    gp = dist.get_global_rank(group, prev) if group is not None else prev
    gn = dist.get_global_rank(group, nxt) if group is not None else nxt
    # tags tell the two directions apart when prev == next (two ranks)
    ops = [dist.P2POp(dist.isend, send_prev, gp, group, tag=1), dist.P2POp(dist.irecv, recv_next, gn, group, tag=1),
           dist.P2POp(dist.isend, send_next, gn, group, tag=2), dist.P2POp(dist.irecv, recv_prev, gp, group, tag=2)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()


class _Band:
    """One band's context and its four packed halo buffers (device memory)."""

    def __init__(self, cfg_global, rank: int, row0: int, own: int, halo: int, device: int):
        import torch
        cfg = cfg_global.copy()
        cfg.ny = own + 2 * halo
        self.rank, self.row0, self.own, self.halo = rank, row0, own, halo
        self.ens = lbl.Ensemble(cfg, device=device)
        self.ens.slab_set(cfg_global.ny, row0, halo)
        nb = self.ens.slab_halo_bytes(halo)
        dev = torch.device("cuda", device)
        self.buf = {k: torch.empty(nb, dtype=torch.uint8, device=dev)
                    for k in ("send_prev", "send_next", "recv_prev", "recv_next")}
        self.torch_stream = torch.cuda.ExternalStream(self.ens.stream(), device=dev)

    def ptr(self, name: str) -> int:
        return self.buf[name].data_ptr()

    def rows(self, ny: int) -> np.ndarray:
        """The global rows of the local rows, halos included."""
        return (self.row0 - self.halo + np.arange(self.own + 2 * self.halo)) % ny


class SlabExperiment:
    """One DA experiment (or nature run) split into y-bands.

    cfg: the whole grid's configuration (lbl.config_default(...)).  With `group` (an
    initialised torch.distributed process group, NCCL for GPUs) this process holds its own
    rank's band on `device`; without it the experiment's `world` bands all live in this
    process on `device` and exchange by reading each other's buffers.  halo: rows kept on each
    side (default_halo(cfg) if None); every band must own at least `halo` rows.  With a group,
    construction, update, assimilate and rmse_uv are collective: every rank calls them in the
    same order (the bands agree on the forecast segment length by an all-reduce at
    construction, and exchange halos in every update and assimilate).
    """

    def __init__(self, cfg, world: int = 1, group=None, halo: Optional[int] = None, device: int = 0,
                 bands: Optional[Sequence[Tuple[int, int]]] = None):
        self.cfg = cfg.copy()
        self.group = group
        if group is not None:
            import torch.distributed as dist
            world, local = dist.get_world_size(group), [dist.get_rank(group)]
        else:
            local = list(range(world))
        self.world, self.nx, self.ny = world, cfg.nx, cfg.ny
        self.halo = default_halo(cfg) if halo is None else int(halo)
        self.bands = list(bands) if bands is not None else partition(cfg.ny, world, row_align(cfg))
        if len(self.bands) != world:
            raise ValueError("one (row0, own) per rank")
        self.local: List[_Band] = []
        try:
            for r in local:
                row0, own = self.bands[r]
                self.local.append(_Band(self.cfg, r, row0, own, self.halo, device))
        except Exception:
            self.close()
            raise
        # every band begins forecasts of the same length: the fewest steps any band's forcing buffer holds
        seg = min(b.ens.slab_forecast_steps() for b in self.local)
        if group is not None and world > 1:
            import torch
            import torch.distributed as dist
            dev = f"cuda:{device}" if dist.get_backend(group) == "nccl" else "cpu"
            t = torch.tensor([seg], dtype=torch.int64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
            seg = int(t.item())
        self.segment = seg

    # -- set-up --------------------------------------------------------------------
    def init(self, ens_offset: int = 0):
        for b in self.local:
            b.ens.init(ens_offset)

    def close(self):
        for b in getattr(self, "local", []):
            b.ens.close()
        self.local = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the exchange --------------------------------------------------------------
    def exchange(self, rows: int):
        """Refresh the outer `rows` rows of every local band from its neighbours."""
        for b in self.local:
            b.ens.slab_pack(rows, b.ptr("send_prev"), b.ptr("send_next"))
        if self.world == 1:
            b = self.local[0]  # its own neighbour on both sides
            b.ens.slab_unpack(rows, b.ptr("send_next"), b.ptr("send_prev"))
            return
        if self.group is not None:
            import torch
            b = self.local[0]
            nb = b.ens.slab_halo_bytes(rows)
            with torch.cuda.stream(b.torch_stream):
                ring_exchange(self.group, b.buf["send_prev"][:nb], b.buf["send_next"][:nb], b.buf["recv_prev"][:nb],
                              b.buf["recv_next"][:nb])
            b.ens.slab_unpack(rows, b.ptr("recv_prev"), b.ptr("recv_next"))
            return
        # every band here: the packs are complete before any neighbour reads them, and the
        # reads before any band packs again
        for b in self.local:
            b.ens.sync()
        for b in self.local:
            prev, nxt = self.local[(b.rank - 1) % self.world], self.local[(b.rank + 1) % self.world]
            b.ens.slab_unpack(rows, prev.ptr("send_next"), nxt.ptr("send_prev"))
        for b in self.local:
            b.ens.sync()

    # -- the cycle ------------------------------------------------------------------
    def update(self, t0: int, nsteps: int):
        """nsteps steps from t0: the forcing of up to `segment` steps at once
        (lbl_slab_forecast_begin), then chunks of halo / 2 steps with an exchange after each."""
        k_max = max(1, self.halo // 2)
        t, left = t0, nsteps
        while left > 0:
            n = min(left, self.segment)
            for b in self.local:
                b.ens.slab_forecast_begin(t, n)
            done = 0
            while done < n:
                k = min(k_max, n - done)
                for b in self.local:
                    b.ens.slab_forecast_chunk(k)
                self.exchange(2 * k)
                done += k
            t += n
            left -= n

    def local_fields(self, b: _Band, *fields):
        """Slices of whole-grid (ny, nx) fields holding band b's rows, halos included."""
        rows = b.rows(self.ny)
        return [np.ascontiguousarray(np.asarray(f, np.float32).reshape(self.ny, self.nx)[rows]) for f in fields]

    def assimilate(self, t: int, rho_o, u_o, v_o):
        """The analysis at step t from whole-grid observation fields, then the halos."""
        for b in self.local:
            ro, uo, vo = self.local_fields(b, rho_o, u_o, v_o)
            b.ens.assimilate(t, ro, uo, vo, sync=False)
        self.exchange(self.halo)

    def sync(self):
        for b in self.local:
            b.ens.sync()

    # -- results ----------------------------------------------------------------------
    def own_f(self, member: int) -> dict:
        """{rank: populations (9, own, nx) of the band's own rows} for the local bands."""
        return {b.rank: b.ens.get_f(member)[:, b.halo:b.halo + b.own] for b in self.local}

    def own_fields(self, member: int) -> dict:
        """{rank: (rho, u, v) of the band's own rows} for the local bands."""
        out = {}
        for b in self.local:
            r, u, v, _ = b.ens.get_fields(member)
            out[b.rank] = tuple(a[b.halo:b.halo + b.own] for a in (r, u, v))
        return out

    def rmse_uv(self, u_true, v_true) -> float:
        """RMSE of the ensemble-mean (u, v) against whole-grid true fields, over the whole
        grid (a collective when the bands are spread over processes)."""
        s = 0.0
        for b in self.local:
            ut, vt = self.local_fields(b, u_true, v_true)
            s += b.ens.rmse_uv(ut, vt) ** 2 * b.own * self.nx
        if self.group is not None and self.world > 1:
            import torch
            import torch.distributed as dist
            dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
            t = torch.tensor([s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, group=self.group)
            s = float(t.item())
        return math.sqrt(s / (self.ny * self.nx))

    def letkf_stats(self) -> dict:
        """Largest sweep count and NaN flag over the local bands (halo points included)."""
        st = [b.ens.letkf_stats() for b in self.local]
        return {"max_sweeps": max(x["max_sweeps"] for x in st), "nan": max(x["nan"] for x in st)}
