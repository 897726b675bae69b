"""z-slab domain decomposition of the periodic box over several ranks.

The reference runs one mesh per process and keeps a halo buffer behind the
owned elements as the landing zone of boundary-face values
(mod_mesh.f90:119-130): mesh_setup gives every face that leaves the domain
consecutive halo slots, and update_halo (mod_mesh.f90:209-221) fills them,
on one process from the periodic source node (halo_src_map).  Split the
NeX x NeY x NeZ box into z-slabs, one per rank, and the x and y faces still
wrap inside the slab, but the -z faces of the bottom layer and the +z faces of
the top layer belong to the neighbouring slabs.  Each RK stage then needs one
exchange: every rank sends the +z face values of its top layer up and the
-z face values of its bottom layer down, Nfp * NeX * NeY values each, and
receives its neighbours' into those halo slots.

Layout.  Rank r owns the element layers [z0, z0 + nz) (the first NeZ mod R
ranks one layer more).  Its local mesh is mesh_setup on NeX x NeY x nz with
domain (1, 1, nz/NeZ): element sizes, normals, Fscale, Escale and every
interior neighbour relation are those of the global mesh, and the local
element e is the global element e0 + e (elements are numbered i + NeX (j +
NeY k), so a z-slab is a contiguous element range).  The local z wraps get
halo slots like any boundary face; after the local update_halo those slots
hold the rank's own opposite layer (its top layer in the -z slots, its bottom
layer in the +z slots), which is exactly what the rank above (below) needs in
its -z (+z) slots.  The exchange is therefore a cyclic shift of those slot
blocks between neighbours, in the (j, i, fp) order in which mesh_setup
numbers them on every rank.

The exchange runs on torch.distributed point-to-point operations (NCCL on
GPUs, gloo on CPU) on whatever tensors hold the stage input, so no data path
goes through a library kernel that is given a peer's memory.
"""
import numpy as np


def slab_range(NeZ, rank, nranks):
    """(z0, nz): the first element layer and the layer count of `rank`."""
    base, extra = divmod(NeZ, nranks)
    nz = base + (1 if rank < extra else 0)
    z0 = rank * base + min(rank, extra)
    return z0, nz


def z_halo_slots(VMapP, Np, Ne, NeX, NeY, nz, Nfp):
    """0-based halo slots of the local -z faces of the bottom layer and the
    +z faces of the top layer, each in (j, i, fp) order (the order in which
    mesh_setup numbers them, mod_mesh.f90:172-190)."""
    VMapP = np.asarray(VMapP).reshape(6 * Nfp, Ne, order="F")
    base = Np * Ne
    lo, hi = [], []
    for j in range(NeY):
        for i in range(NeX):
            eb = i + NeX * j                       # bottom layer, local k = 0
            et = i + NeX * (j + NeY * (nz - 1))    # top layer
            lo.append(VMapP[4 * Nfp: 5 * Nfp, eb] - 1 - base)
            hi.append(VMapP[5 * Nfp: 6 * Nfp, et] - 1 - base)
    lo = np.concatenate(lo).astype(np.int64)
    hi = np.concatenate(hi).astype(np.int64)
    if lo.min() < 0 or hi.min() < 0:
        raise ValueError("z faces of the slab do not lead into the halo")
    return lo, hi


class ZSlab:
    """One rank's slab: its element range in the global box, its local mesh
    tables (from the library's mesh_setup or the oracle's, both
    bit-identical to the reference's) and its z halo slots."""

    def __init__(self, NeX, NeY, NeZ, p, x1D, rank, nranks, mesh_setup):
        self.NeX, self.NeY, self.NeZ, self.p = NeX, NeY, NeZ, p
        self.rank, self.nranks = rank, nranks
        self.z0, self.nz = slab_range(NeZ, rank, nranks)
        if self.nz < 1:
            raise ValueError(f"rank {rank} of {nranks} gets no element layer of {NeZ}")
        self.mesh = mesh_setup(NeX, NeY, self.nz, p, x1D, (1.0, 1.0, self.nz / NeZ))
        m = self.mesh
        self.Nfp = (p + 1) ** 2
        self.e0 = self.z0 * NeX * NeY          # first global element
        self.lo, self.hi = z_halo_slots(m.VMapP, m.Np, m.Ne, NeX, NeY, self.nz, self.Nfp)

    @property
    def up(self):
        return (self.rank + 1) % self.nranks

    @property
    def down(self):
        return (self.rank - 1) % self.nranks

    def local(self, global_field):
        """This rank's owned columns (Np, Ne) of a global (Np, >= Ne_g) field,
        as a new (Np, NeA) array with an empty halo."""
        m = self.mesh
        g = np.asarray(global_field).reshape(m.Np, -1, order="F")
        out = np.zeros((m.Np, m.NeA), order="F", dtype=g.dtype)
        out[:, : m.Ne] = g[:, self.e0: self.e0 + m.Ne]
        return out

    def _slots(self, device):
        import torch
        key = str(device)
        if getattr(self, "_slot_dev", None) != key:
            base = self.mesh.Np * self.mesh.Ne
            self._lo_t = torch.as_tensor(base + self.lo, device=device)
            self._hi_t = torch.as_tensor(base + self.hi, device=device)
            self._slot_dev = key
        return self._lo_t, self._hi_t

    def pack(self, f_flat):
        """The blocks this rank sends, from the flat stage array `f_flat` (a
        torch tensor holding the local update_halo): (to the rank above: my
        top layer's +z face nodes, to the rank below: my bottom layer's -z
        face nodes)."""
        lo_t, hi_t = self._slots(f_flat.device)
        return f_flat.index_select(0, lo_t), f_flat.index_select(0, hi_t)

    def unpack(self, f_flat, from_below, from_above):
        """Writes the blocks received from the ranks below and above into the
        -z and +z halo slots of `f_flat`."""
        lo_t, hi_t = self._slots(f_flat.device)
        f_flat.index_copy_(0, lo_t, from_below)
        f_flat.index_copy_(0, hi_t, from_above)

    def exchange(self, f_flat, dist, make_tensor):
        """Fills the z halo slots of the flat stage array `f_flat` (a torch
        tensor, already holding the local update_halo) with the neighbours'
        boundary layers.  `make_tensor(n)` allocates a receive buffer like
        f_flat.  Every rank makes the same calls in the same order."""
        if self.nranks == 1:
            return  # the local update_halo is already the periodic wrap
        send_up, send_dn = self.pack(f_flat)
        recv_dn = make_tensor(self.lo.size)
        recv_up = make_tensor(self.hi.size)
        # Tag 1: traffic going up (to rank + 1), tag 2: going down.
        ops = [dist.P2POp(dist.isend, send_up, self.up, tag=1),
               dist.P2POp(dist.irecv, recv_dn, self.down, tag=1),
               dist.P2POp(dist.isend, send_dn, self.down, tag=2),
               dist.P2POp(dist.irecv, recv_up, self.up, tag=2)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        self.unpack(f_flat, recv_dn, recv_up)


def exchange_local(slabs, arrays):
    """The exchange of all ranks' slabs held by one process (one GPU): the
    blocks each slab would send go straight into its neighbours' halo
    slots.  arrays[r] is slab r's flat stage array."""
    out = [sl.pack(a) for sl, a in zip(slabs, arrays)]
    for sl, a in zip(slabs, arrays):
        sl.unpack(a, out[sl.down][0], out[sl.up][1])
