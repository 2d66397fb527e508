"""Exchanges of a solve whose panels are split across ranks.

Two lists move values between panels during a stage, and both are explicit:

* the ghost fill (cs_fill_ghosts; cs_fill_map_get): each entry sets one
  ghost value from one source value (source and destination offsets into
  the field arrays, the fields, a sign, and whether the value is averaged
  with the destination's own).  This is the exchange of the reference's
  LOAD_LOCAL_BUFFERS_* / FETCH_BUFFERS_FILL_IN_* routines
  (300riemann_module/320-333), which run it between MPI ranks that each own
  panels;
* panel-edge ownership (cs_sync_map_get): the face fluxes and edge EMFs that
  two or three panels compute take the lowest-numbered panel's value, the
  single-device form of the reference's defect exchange (DRV:3200-3461).

With the panels assigned to ranks, the entries whose destination panel a
rank owns split into those it can apply from its own panels and those whose
source panel another rank owns; every rank derives both its receive lists
and the matching send lists from the same global list, so the two sides
agree on order without exchanging any index.  Host arrays (numpy) hold the
fields for the single-process forms; torch tensors (CPU with gloo, CUDA with
NCCL) for the split ones, one grouped point-to-point round per exchange.
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


def apply_face_sync(fcon, EF, dst, src, dk, sk) -> None:
    """Face ownership on host arrays, in place: fcon[d] (2m, 6 * box) holds
    a direction's two one-sided contributions (rows 0..m-1 and m..2m-1; m = 8
    on the device) and EF[d] (6 * box) its entropy flux; each listed copy
    takes its owner's contributions with the sides exchanged and the negated
    entropy flux."""
    for d in range(len(fcon)):
        for s in range(len(fcon)):
            sel = np.flatnonzero((dk == d) & (sk == s))
            if len(sel):
                fcon[d][:, dst[sel]] = np.roll(fcon[s][:, src[sel]], fcon[s].shape[0] // 2, axis=0)
                EF[d][dst[sel]] = -EF[s][src[sel]]


def apply_edge_sync(Ef, dst, src, dk, sk, sign) -> None:
    """Edge ownership on host arrays, in place: Ef[c] (6 * box) is EMF
    component c; each listed copy takes its owner's value times sign."""
    vals = np.array([sign[t] * Ef[sk[t]][src[t]] for t in range(len(dst))])
    for c in range(len(Ef)):
        sel = dk == c
        Ef[c][dst[sel]] = vals[sel]


def apply_face_average(fcon, EF, dst, src, dk, sk) -> None:
    """The reference's rule for shared faces (CS_FLAG_PANEL_AVERAGE) on host
    arrays laid out as for apply_face_sync, in place: both copies of each
    listed face take the average of the two panels' contributions (sides
    exchanged) and of their entropy fluxes (negated), as k_avg_flux does."""
    for d in range(len(fcon)):
        for s in range(len(fcon)):
            sel = np.flatnonzero((dk == d) & (sk == s))
            if len(sel):
                m = fcon[d].shape[0] // 2
                own, other = fcon[d][:, dst[sel]], np.roll(fcon[s][:, src[sel]], m, axis=0)
                avg = (own + other) * 0.5
                fcon[d][:, dst[sel]] = avg
                fcon[s][:, src[sel]] = np.roll(avg, m, axis=0)
                e = (EF[d][dst[sel]] - EF[s][src[sel]]) * 0.5
                EF[d][dst[sel]] = e
                EF[s][src[sel]] = -e


def edge_classes(src, sk):
    """Starts of the runs of entries that share an owner copy (one run an
    edge: one entry for an edge of two panels, two at a cube corner), then
    the entry count; the device builds the same starts with the list."""
    key = sk.astype(np.int64) << 40 | src.astype(np.int64)
    return np.concatenate([[0], np.flatnonzero(key[1:] != key[:-1]) + 1, [len(src)]])


def apply_edge_average(Ef, dst, src, dk, sk, sign) -> None:
    """The reference's rule for shared edges (CS_FLAG_PANEL_AVERAGE) on host
    arrays Ef[c] (6 * box), in place: every copy takes the signed average of
    the copies, (own + other) * 0.5 for two and their sum / 3 for the three of
    a cube-corner radial edge, as k_avg_emf does."""
    cls = edge_classes(src, sk)
    for q in range(len(cls) - 1):
        h, n = cls[q], cls[q + 1] - cls[q]
        total = Ef[sk[h]][src[h]]
        for m in range(h, h + n):
            total = total + float(sign[m]) * Ef[dk[m]][dst[m]]
        avg = total * 0.5 if n == 1 else total / 3.0
        Ef[sk[h]][src[h]] = avg
        for m in range(h, h + n):
            Ef[dk[m]][dst[m]] = float(sign[m]) * avg


class PanelSplit:
    """Entries of one exchange list as one rank sees them: `panel_rank[p]`
    is the rank owning panel p, `box` the points of one panel box, and src /
    dst the entries' offsets (for multi-component fields, any offset whose
    panel is (offset // box) % 6).  `mine` are the entries whose destination
    panel this rank owns: `local` ones from its own panels, the `recv[q]`
    ones from values rank q sends, in the global list's order; `send[q]`
    lists the entries rank q applies from this rank's panels, in the same
    order."""

    def __init__(self, src, dst, box: int, panel_rank, rank: int):
        panel_rank = np.asarray(panel_rank)
        self.src, self.dst = np.asarray(src), np.asarray(dst)
        sp = panel_rank[(self.src // box) % 6]
        dp = panel_rank[(self.dst // box) % 6]
        self.rank = rank
        self.peers = sorted(set(int(r) for r in panel_rank) - {rank})
        self.mine = np.flatnonzero(dp == rank)
        self.local = np.flatnonzero((dp == rank) & (sp == rank))
        self.recv = {q: np.flatnonzero((dp == rank) & (sp == q)) for q in self.peers}
        self.send = {q: np.flatnonzero((dp == q) & (sp == rank)) for q in self.peers}

    def values_bytes(self, width: int = 1) -> int:
        """Bytes this rank sends per exchange (`width` FP64 values an entry)."""
        return 8 * width * sum(len(v) for v in self.send.values())

    def route(self, gather, dist, width: int, device):
        """Source values of every entry in `mine` (a (len(mine), width) FP64
        tensor, in `mine`'s order): `gather(entries)` reads the values of
        the given entries from this rank's panels; every source value is
        read before the caller writes any destination.  Every rank of the
        split calls it together."""
        import torch

        bufs = {q: gather(self.send[q]) for q in self.peers}
        incoming = {q: torch.empty((len(self.recv[q]), width), dtype=torch.float64, device=device) for q in self.peers}
        ops = []
        for q in self.peers:
            if len(self.send[q]):
                ops.append(dist.P2POp(dist.isend, bufs[q].contiguous(), q))
            if len(self.recv[q]):
                ops.append(dist.P2POp(dist.irecv, incoming[q], q))
        for w in (dist.batch_isend_irecv(ops) if ops else []):
            w.wait()
        vals = torch.empty((len(self.src), width), dtype=torch.float64, device=device)
        vals[torch.as_tensor(self.local, device=device, dtype=torch.long)] = gather(self.local)
        for q in self.peers:
            vals[torch.as_tensor(self.recv[q], device=device, dtype=torch.long)] = incoming[q]
        return vals[torch.as_tensor(self.mine, device=device, dtype=torch.long)]


def _idx(a, dev):
    import torch

    return torch.as_tensor(a, device=dev, dtype=torch.long)


class GhostExchange(PanelSplit):
    """The ghost fill split across ranks (cs_fill_map_get's src, dst, meta)."""

    def __init__(self, src, dst, meta, box: int, panel_rank, rank: int):
        super().__init__(src, dst, box, panel_rank, rank)
        self.meta = np.asarray(meta)

    def exchange(self, st: dict, dist) -> None:
        """Fills this rank's ghost values in `st` (torch tensors U, ent,
        bxf, byf, bzf; the other ranks' panels may hold anything) from its
        own panels and its peers' messages."""
        import torch

        flat = _fields(st)
        dev = flat[0].device

        def gather(entries):
            s, f = self.src[entries], self.meta[entries] >> 5
            out = torch.empty((len(entries), 1), dtype=torch.float64, device=dev)
            for k in range(5):
                sel = np.flatnonzero(f == k)
                if len(sel):
                    out[_idx(sel, dev), 0] = flat[k][_idx(s[sel], dev)].to(torch.float64)
            return out

        v = self.route(gather, dist, 1, dev)[:, 0]
        d, m = self.dst[self.mine], self.meta[self.mine]
        old = torch.empty(len(d), dtype=torch.float64, device=dev)
        for k in range(5):
            sel = np.flatnonzero((m & 7) == k)
            if len(sel):
                old[_idx(sel, dev)] = flat[k][_idx(d[sel], dev)].to(torch.float64)
        v = _finish(v, m, old)
        for k in range(5):
            sel = np.flatnonzero((m & 7) == k)
            if len(sel):
                flat[k][_idx(d[sel], dev)] = v[_idx(sel, dev)].to(flat[k].dtype)


class FaceSync(PanelSplit):
    """Face ownership split across ranks (cs_sync_map_get(0)): ncomp + 1
    values an entry, the owner's one-sided contributions (ncomp / 2 a side:
    8 on the device, whose face arrays hold one value a variable and side)
    and its entropy flux."""

    def __init__(self, dst, src, dk, sk, box: int, panel_rank, rank: int, ncomp: int = 16):
        super().__init__(src, dst, box, panel_rank, rank)
        self.dk, self.sk = np.asarray(dk), np.asarray(sk)
        self.ncomp = ncomp

    def exchange(self, fcon, EF, dist) -> None:
        """fcon[d]: (ncomp, 6 * box) torch tensors (one side's rows, then the
        other's), EF[d]: (6 * box), d the face direction; this rank's listed
        copies take their owners' values (sides exchanged, entropy flux
        negated)."""
        import torch

        dev = EF[0].device
        m = self.ncomp

        def gather(entries):
            out = torch.empty((len(entries), m + 1), dtype=torch.float64, device=dev)
            s, k = self.src[entries], self.sk[entries]
            for d in range(len(fcon)):
                sel = np.flatnonzero(k == d)
                if len(sel):
                    out[_idx(sel, dev), :m] = fcon[d][:, _idx(s[sel], dev)].T.to(torch.float64)
                    out[_idx(sel, dev), m] = EF[d][_idx(s[sel], dev)].to(torch.float64)
            return out

        v = self.route(gather, dist, m + 1, dev)
        d, k = self.dst[self.mine], self.dk[self.mine]
        for q in range(len(fcon)):
            sel = np.flatnonzero(k == q)
            if len(sel):
                rows = v[_idx(sel, dev)]
                fcon[q][:, _idx(d[sel], dev)] = torch.roll(rows[:, :m], m // 2, dims=1).T.to(fcon[q].dtype)
                EF[q][_idx(d[sel], dev)] = (-rows[:, m]).to(EF[q].dtype)


class EdgeSync(PanelSplit):
    """Edge ownership split across ranks (cs_sync_map_get(1))."""

    def __init__(self, dst, src, dk, sk, sign, box: int, panel_rank, rank: int):
        super().__init__(src, dst, box, panel_rank, rank)
        self.dk, self.sk, self.sign = np.asarray(dk), np.asarray(sk), np.asarray(sign)

    def exchange(self, Ef, dist) -> None:
        """Ef[c]: (6 * box) torch tensors, c the EMF component; this rank's
        listed copies take their owners' values times the sign."""
        import torch

        dev = Ef[0].device

        def gather(entries):
            out = torch.empty((len(entries), 1), dtype=torch.float64, device=dev)
            s, k = self.src[entries], self.sk[entries]
            for c in range(len(Ef)):
                sel = np.flatnonzero(k == c)
                if len(sel):
                    out[_idx(sel, dev), 0] = Ef[c][_idx(s[sel], dev)].to(torch.float64)
            return out

        v = self.route(gather, dist, 1, dev)[:, 0]
        v = v * torch.as_tensor(self.sign[self.mine], device=dev, dtype=torch.float64)
        d, k = self.dst[self.mine], self.dk[self.mine]
        for c in range(len(Ef)):
            sel = np.flatnonzero(k == c)
            if len(sel):
                Ef[c][_idx(d[sel], dev)] = v[_idx(sel, dev)].to(Ef[c].dtype)
