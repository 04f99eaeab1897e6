"""Row bands of one 2D domain over several ranks, one GPU each.

The reference's multi-GPU program (fun_multi.cu:281-289, 532-533) splits the
periodic j axis of one domain into contiguous bands and, per step, gathers and
scatters whole fields through the host.  Here each rank steps its own band
with rs_step in band mode (rs_params.band = 1: ghost rows supplied by the
caller, interface noise keyed by the global row) and, per step, swaps one edge
row of psi and c with each neighbour: the band's first interior row becomes
the previous band's bottom ghost row, its last interior row the next band's
top ghost row (wrapping around for periodic j).  The moving frame needs the
global coarse tip (a max over ranks) and the solute mass a sum over ranks.

The exchange is torch.distributed point-to-point (NCCL between GPUs, gloo for
CPU tensors); with one rank, or with all bands on one device, it reduces to
local row copies.
"""
from . import _abi


def split_rows(nj, world):
    """Interior rows 1..nj split into `world` contiguous bands: [(first, last)]."""
    base, extra = divmod(nj, world)
    out, a = [], 1
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((a, a + n - 1))
        a += n
    return out


def band_params(p, rank, world):
    """The rs_params of one band: global rows first-1 .. last+1 (two ghost rows)."""
    nj = p.ny_all - 2
    if world < 1 or nj < 6 * world:
        raise ValueError(f"{nj} interior rows cannot form {world} bands of at least 6 rows")
    first, last = split_rows(nj, world)[rank]
    q = _abi.Params.from_buffer_copy(p)
    q.ny_all = last - first + 3
    q.j_offset = first - 1
    q.band = 1
    return q


def _edges(f):
    """(first interior row, last interior row, top ghost row, bottom ghost row) views."""
    return f[1], f[-2], f[0], f[-1]


def exchange(fields, rank, world, periodic=True, group=None):
    """Fills the ghost rows of this band's fields (a list of 2D tensors, rows
    contiguous) from the neighbouring bands; every rank calls it at the same
    point of the step."""
    import torch.distributed as dist
    if world == 1:
        for f in fields:
            first, last, top, bottom = _edges(f)
            if periodic:
                top.copy_(last)
                bottom.copy_(first)
            else:
                top.copy_(first)
                bottom.copy_(last)
        return
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    has_prev = periodic or rank > 0
    has_next = periodic or rank < world - 1
    # Messages between two ranks match in the order they are posted (NCCL
    # has no tags), so every rank posts, per field, "last row down, top
    # ghost from above" and then "first row up, bottom ghost from below";
    # with two ranks the one peer is both neighbours and the orders agree.
    ops = []
    for f in fields:
        first, last, top, bottom = _edges(f)
        if has_next:
            ops.append(dist.P2POp(dist.isend, last, nxt, group))
        if has_prev:
            ops.append(dist.P2POp(dist.irecv, top, prev, group))
        if has_prev:
            ops.append(dist.P2POp(dist.isend, first, prev, group))
        if has_next:
            ops.append(dist.P2POp(dist.irecv, bottom, nxt, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for f in fields:  # no-flux ends of a non-periodic axis
        first, last, top, bottom = _edges(f)
        if not has_prev:
            top.copy_(first)
        if not has_next:
            bottom.copy_(last)


def exchange_local(band_fields, periodic=True):
    """The same exchange for bands that live on one device (or host): a list,
    in band order, of each band's list of fields."""
    n = len(band_fields)
    for r, fields in enumerate(band_fields):
        prev, nxt = (r - 1) % n, (r + 1) % n
        for k, f in enumerate(fields):
            _, _, top, bottom = _edges(f)
            if periodic or r > 0:
                top.copy_(band_fields[prev][k][-2])
            else:
                top.copy_(f[1])
            if periodic or r < n - 1:
                bottom.copy_(band_fields[nxt][k][1])
            else:
                bottom.copy_(f[-2])


class Band:
    """One rank's band of a 2D domain: its context, two field sets and the
    per-step exchange.  `step` follows the reference loop body (main.cu
    order): the pull-back decision from the global coarse tip, the step, then
    the ghost rows of the new fields."""

    def __init__(self, p, rank, world, dtype, group=None):
        from . import lib
        self.p_global, self.rank, self.world, self.group = p, rank, world, group
        self.p = band_params(p, rank, world)
        self.ctx = lib.Context(self.p)
        self.d = self.ctx.d
        self.cur, self.nxt = lib.FieldSet(self.p, dtype), lib.FieldSet(self.p, dtype)
        self.periodic = bool(p.periodic_j)

    def exchange(self, fs):
        exchange([fs.psi, fs.c], self.rank, self.world, self.periodic, self.group)

    def initial_planar(self, c_liquid, c_solid, seed):
        self.ctx.initial_planar(self.cur, c_liquid, c_solid, seed)
        self.exchange(self.cur)

    def global_itip(self, itip):
        """rs_itip over the band, then the max over ranks (get_itip_all_grain)."""
        import torch.distributed as dist
        self.ctx.itip(self.cur, itip)
        if self.world > 1:
            dist.all_reduce(itip, op=dist.ReduceOp.MAX, group=self.group)
        return itip

    def global_mass(self, out):
        import torch.distributed as dist
        self.ctx.mass(self.cur, out)
        if self.world > 1:
            dist.all_reduce(out, op=dist.ReduceOp.SUM, group=self.group)
        return out

    def step(self, n, i_offset_history=0, l_offset_Vp=0.0, pull_back=None):
        self.ctx.step(self.cur, self.nxt, n, i_offset_history=i_offset_history, l_offset_Vp=l_offset_Vp,
                      pull_back=pull_back)
        self.cur, self.nxt = self.nxt, self.cur
        self.exchange(self.cur)
