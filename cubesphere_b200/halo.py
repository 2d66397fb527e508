"""Ghost exchange of a solve whose panels are split across ranks.

The device fill (cs_fill_ghosts) applies one list of entries, each setting
one ghost value from one source value (cs_fill_map_get: source and
destination offsets into the field arrays, the fields, a sign, and whether
the value is averaged with the destination's own).  This is the exchange of
the reference's LOAD_LOCAL_BUFFERS_* / FETCH_BUFFERS_FILL_IN_* routines
(300riemann_module/320-333), which run it between MPI ranks that each own
panels.  With the panels assigned to ranks, the entries whose destination
panel a rank owns split into those it can apply from its own panels and
those whose source panel another rank owns; every rank derives both its
receive lists and the matching send lists from the same global list, so the
two sides agree on order without exchanging any index.

Host arrays or torch tensors (CPU with gloo, CUDA with NCCL) hold the
fields; `exchange` is one grouped point-to-point round per call.
"""
from __future__ import annotations

import numpy as np

FIELDS = ("U", "ent", "bxf", "byf", "bzf")


def _fields(st):
    return [st[k].reshape(-1) for k in FIELDS]


def _finish(vals, meta, old):
    """Sign, then the average with the destination's pre-exchange value."""
    neg = (meta & 8) != 0
    vals = np.where(neg, -vals, vals) if isinstance(vals, np.ndarray) else _torch_where(neg, -vals, vals)
    avg = (meta & 16) != 0
    if avg.any():
        if isinstance(vals, np.ndarray):
            vals = np.where(avg, (old + vals) * 0.5, vals)
        else:
            vals = _torch_where(avg, (old + vals) * 0.5, vals)
    return vals


def _torch_where(mask, a, b):
    import torch

    return torch.where(torch.as_tensor(mask, device=a.device), a, b)


def apply_fill_map(st: dict, src, dst, meta) -> None:
    """The whole ghost exchange on host arrays `st` (U, ent, bxf, byf, bzf
    in the panel-box layout), in place: every source value is read before
    any destination is written, as on the device."""
    flat = _fields(st)
    sf, df = meta >> 5, meta & 7
    vals = np.empty(len(src))
    old = np.empty(len(src))
    for f in range(5):
        sel = sf == f
        vals[sel] = flat[f][src[sel]]
        sel = df == f
        old[sel] = flat[f][dst[sel]]
    vals = _finish(vals, meta, old)
    for f in range(5):
        sel = df == f
        flat[f][dst[sel]] = vals[sel]


class PanelSplit:
    """Exchange lists of one rank: `panel_rank[p]` is the rank owning panel
    p; `box` the points of one panel box.  Entries whose destination panel
    this rank owns are applied here: `local` ones from its own panels, the
    `recv[q]` ones from values rank q sends, in the global list's order;
    `send[q]` lists the entries rank q applies from this rank's panels, in
    the same order."""

    def __init__(self, src, dst, meta, box: int, panel_rank, rank: int):
        panel_rank = np.asarray(panel_rank)
        self.src, self.dst, self.meta = np.asarray(src), np.asarray(dst), np.asarray(meta)
        sp = panel_rank[(self.src // box) % 6]
        dp = panel_rank[(self.dst // box) % 6]
        self.rank = rank
        self.peers = sorted(set(int(r) for r in panel_rank) - {rank})
        self.mine = np.flatnonzero(dp == rank)
        self.local = np.flatnonzero((dp == rank) & (sp == rank))
        self.recv = {q: np.flatnonzero((dp == rank) & (sp == q)) for q in self.peers}
        self.send = {q: np.flatnonzero((dp == q) & (sp == rank)) for q in self.peers}

    def values_bytes(self) -> int:
        """Bytes this rank sends per exchange (FP64 values)."""
        return 8 * sum(len(v) for v in self.send.values())

    def exchange(self, st: dict, dist) -> None:
        """Fills this rank's ghost values in `st` (torch tensors; the other
        ranks' panels may hold anything) from its own panels and its peers'
        messages; every rank of the split calls it together."""
        import torch

        flat = _fields(st)
        dev = flat[0].device
        idx = lambda a: torch.as_tensor(a, device=dev, dtype=torch.long)

        def gather(entries):
            s, f = self.src[entries], self.meta[entries] >> 5
            out = torch.empty(len(entries), dtype=torch.float64, device=dev)
            for k in range(5):
                sel = np.flatnonzero(f == k)
                if len(sel):
                    out[idx(sel)] = flat[k][idx(s[sel])].to(torch.float64)
            return out

        # every source value read before any destination is written
        bufs = {q: gather(self.send[q]) for q in self.peers}
        incoming = {q: torch.empty(len(self.recv[q]), dtype=torch.float64, device=dev) for q in self.peers}
        ops = []
        for q in self.peers:
            if len(self.send[q]):
                ops.append(dist.P2POp(dist.isend, bufs[q], q))
            if len(self.recv[q]):
                ops.append(dist.P2POp(dist.irecv, incoming[q], q))
        for w in (dist.batch_isend_irecv(ops) if ops else []):
            w.wait()
        vals = torch.empty(len(self.src), dtype=torch.float64, device=dev)
        vals[idx(self.local)] = gather(self.local)
        for q in self.peers:
            vals[idx(self.recv[q])] = incoming[q]
        mine = self.mine
        d, m = self.dst[mine], self.meta[mine]
        old = torch.empty(len(mine), dtype=torch.float64, device=dev)
        for k in range(5):
            sel = np.flatnonzero((m & 7) == k)
            if len(sel):
                old[idx(sel)] = flat[k][idx(d[sel])].to(torch.float64)
        v = _finish(vals[idx(mine)], m, old)
        for k in range(5):
            sel = np.flatnonzero((m & 7) == k)
            if len(sel):
                flat[k][idx(d[sel])] = v[idx(sel)].to(flat[k].dtype)
