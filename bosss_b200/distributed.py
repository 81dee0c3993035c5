"""Partitioned evaluation over several GPUs: x-slab domain decomposition with ghost layers.

The reference evaluates a partitioned grid with one MPI process per part: before the
volume pass it starts the exchange of the DG coefficients of the face neighbours that
live on other processes (``Transceiver.cs:198-250``), evaluates, and finishes the exchange
before the cells that need it (``DifferentialOperator.cs:1599-1627``). Here every rank owns
one GPU and a contiguous slab of x-planes of a uniform Cartesian grid (generator cell order,
x slowest, so a slab is one contiguous range of the global coefficient vector):

* :class:`SlabPartition` -- which planes a rank owns, its ghost planes, the part's grid
  descriptor (the owned planes plus one ghost plane per side that is not a global boundary;
  ``global_n``/``global_offset``/``global_periodic`` let the SIP penalty see the global
  boundary), and the cell ranges of the interior and of the planes next to the ghosts;
* :class:`HaloExchange` -- the exchange of the first/last owned plane into the neighbours'
  ghost planes with ``torch.distributed`` point-to-point operations (NCCL over NVLink between
  GPUs, gloo between CPU processes); ghost planes are received directly into the part's
  vector, no packing;
* :class:`PartEvaluator` -- the device evaluator of one part (``bosss_b200_create`` with the
  part's grid descriptor, ``bosss_b200_apply_device`` on cell ranges);
* :class:`DistributedEvaluator` -- residual / JVP / VJP of the partitioned operator: the halo
  exchange is started, the interior cells are evaluated while it is in flight, then the
  planes next to the ghosts.

Vectors are part vectors (ghost planes included); :meth:`SlabPartition.own` is the view of
the owned DOFs, which are exactly the rank's slice of the global vector.
"""
import ctypes

import numpy as np

from . import _capi as C
from .operator import CartesianGrid, np_of


class SlabPartition:
    """x-slab partition of ``grid`` over ``nranks`` ranks (planes split as evenly as possible)."""

    def __init__(self, grid, nranks, rank, dofs_per_cell):
        if grid.cell_order != C.CELLS_GENERATOR:
            raise ValueError("slab partitions need the generator cell order (x slowest)")
        nx = grid.n[0]
        if not (1 <= nranks <= nx) or not (0 <= rank < nranks):
            raise ValueError("need 1 <= nranks <= number of x-planes and 0 <= rank < nranks")
        self.grid, self.nranks, self.rank = grid, nranks, rank
        base, extra = divmod(nx, nranks)
        counts = [base + (1 if r < extra else 0) for r in range(nranks)]
        self.first = sum(counts[:rank])
        self.count = counts[rank]
        per = bool(grid.periodic[0])
        multi = nranks > 1
        self.ghost_lo = int(multi and (self.first > 0 or per))
        self.ghost_hi = int(multi and (self.first + self.count < nx or per))
        self.left = (rank - 1) % nranks if self.ghost_lo else None
        self.right = (rank + 1) % nranks if self.ghost_hi else None
        self.plane_cells = int(np.prod(grid.n[1:]))
        self.dofs_per_cell = int(dofs_per_cell)
        self.plane_dofs = self.plane_cells * self.dofs_per_cell
        self.n_planes = self.count + self.ghost_lo + self.ghost_hi
        self.n_cells = self.n_planes * self.plane_cells
        self.n_dofs = self.n_cells * self.dofs_per_cell

    # ---- grid of the part
    def grid_desc(self):
        """``bosss_grid_desc`` of the part: owned planes plus ghost planes."""
        g = self.grid
        x0 = self.first - self.ghost_lo
        d = C.GridDesc()
        d.dim = g.dim
        for k in range(3):
            d.n[k] = g.n[k] if k < g.dim else 1
            d.lo[k] = g.lo[k] if k < g.dim else 0.0
            d.hi[k] = g.hi[k] if k < g.dim else 1.0
            d.periodic[k] = int(g.periodic[k]) if k < g.dim else 0
        d.cell_order = C.CELLS_GENERATOR
        if self.nranks > 1:
            # lo/hi stay the global box: the library derives the global cell width from it
            d.n[0] = self.n_planes
            d.periodic[0] = 0
            for k in range(g.dim):
                d.global_n[k] = g.n[k]
                d.global_periodic[k] = int(g.periodic[k])
            d.global_offset[0] = x0
        return d

    # ---- ranges (cells of the part's grid)
    def own_cells(self):
        return self.ghost_lo * self.plane_cells, (self.ghost_lo + self.count) * self.plane_cells

    def interior_cells(self):
        """Owned cells none of whose face neighbours is a ghost cell (may be empty)."""
        lo = self.ghost_lo + (1 if self.ghost_lo else 0)
        hi = self.ghost_lo + self.count - (1 if self.ghost_hi else 0)
        hi = max(hi, lo)
        return lo * self.plane_cells, hi * self.plane_cells

    def rim_cells(self):
        """Cell ranges of the owned planes next to a ghost plane (the owned cells outside
        :meth:`interior_cells`)."""
        own0, own1 = self.own_cells()
        in0, in1 = self.interior_cells()
        if in1 <= in0:
            return [(own0, own1)]
        return [(a, b) for a, b in ((own0, in0), (in1, own1)) if b > a]

    # ---- views of a part vector
    def own(self, x):
        a, b = self.own_cells()
        return x[a * self.dofs_per_cell:b * self.dofs_per_cell]

    def first_plane(self, x):
        o = self.ghost_lo * self.plane_dofs
        return x[o:o + self.plane_dofs]

    def last_plane(self, x):
        o = (self.ghost_lo + self.count - 1) * self.plane_dofs
        return x[o:o + self.plane_dofs]

    def ghost_lo_plane(self, x):
        return x[0:self.plane_dofs] if self.ghost_lo else None

    def ghost_hi_plane(self, x):
        o = (self.ghost_lo + self.count) * self.plane_dofs
        return x[o:o + self.plane_dofs] if self.ghost_hi else None

    def global_slice(self):
        """Slice of the global vector owned by this rank."""
        return slice(self.first * self.plane_dofs, (self.first + self.count) * self.plane_dofs)

    def from_global(self, x_global):
        """Part vector (ghosts included) cut from a global vector: what the halo exchange
        delivers, computed locally (initial data, tests)."""
        nx = self.grid.n[0]
        P = self.plane_dofs
        planes = [(self.first - self.ghost_lo + i) % nx for i in range(self.n_planes)]
        parts = [x_global[p * P:(p + 1) * P] for p in planes]
        if isinstance(x_global, np.ndarray):
            return np.concatenate(parts)
        import torch
        return torch.cat(parts)


class HaloExchange:
    """Ghost-plane exchange of a part vector with ``torch.distributed`` point-to-point ops.

    Every rank posts its sends in the order (last owned plane -> right neighbour, first owned
    plane -> left neighbour) and its receives in the order (left ghost <- left neighbour,
    right ghost <- right neighbour); with two ranks on a periodic grid both neighbours are the
    same rank and this order pairs the planes correctly."""

    def __init__(self, part, group=None):
        self.part, self.group = part, group

    def _peer(self, r):
        import torch.distributed as dist
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def start(self, *vectors):
        """Post the exchange of the ghost planes of every vector; returns the requests."""
        import torch.distributed as dist
        p = self.part
        if p.nranks == 1:
            return []
        ops = []
        for x in vectors:
            if p.right is not None:
                ops.append(dist.P2POp(dist.isend, p.last_plane(x), self._peer(p.right), self.group))
            if p.left is not None:
                ops.append(dist.P2POp(dist.isend, p.first_plane(x), self._peer(p.left), self.group))
            if p.left is not None:
                ops.append(dist.P2POp(dist.irecv, p.ghost_lo_plane(x), self._peer(p.left), self.group))
            if p.right is not None:
                ops.append(dist.P2POp(dist.irecv, p.ghost_hi_plane(x), self._peer(p.right), self.group))
        return dist.batch_isend_irecv(ops) if ops else []

    @staticmethod
    def wait(reqs):
        for r in reqs:
            r.wait()

    def exchange(self, *vectors):
        self.wait(self.start(*vectors))


class PartEvaluator:
    """Device evaluator of one part (``bosss_b200_create`` on the part's grid descriptor)."""

    def __init__(self, op, grid, dom_deg, cod_deg, part, device=0, kernel=C.KERNEL_AUTO):
        self.handle = None
        self.part = part
        self.desc = op.descriptor(dom_deg, cod_deg, grid.dim)
        self.gdesc = part.grid_desc()
        opt = C.Options()
        opt.device, opt.kernel = int(device), int(kernel)
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_create(ctypes.byref(self.desc), ctypes.byref(self.gdesc), ctypes.byref(opt),
                                          ctypes.byref(h)))
        self.handle = h
        nd, nc, nq = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        C.check(C.lib().bosss_b200_get_sizes(h, ctypes.byref(nd), ctypes.byref(nc), ctypes.byref(nq)))
        if nd.value != part.n_dofs or nc.value != part.n_dofs:
            raise ValueError("partitioned evaluation needs a square operator with the part's DOF count")

    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_destroy(self.handle)
            self.handle = None

    __del__ = Dispose

    @staticmethod
    def _stream():
        import torch
        s = torch.cuda.current_stream().cuda_stream
        return ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)

    def apply(self, mode, U, V, out, cells, alpha=1.0, beta=0.0, time=0.0):
        """Residual ``out = beta*out + alpha*Op(U)``, or the JVP / VJP product (alpha, beta unused),
        on the cell range ``cells`` (CUDA tensors)."""
        a, b = cells
        C.check(C.lib().bosss_b200_apply_device(self.handle, int(mode), float(alpha), float(beta), C.ptr(U),
                                                C.ptr(V), C.ptr(out), float(time), int(a), int(b), self._stream()))


class DistributedEvaluator:
    """Residual / JVP / VJP of an operator on a grid partitioned into x-slabs, one rank per GPU.

    ``op``: committed :class:`~bosss_b200.operator.DifferentialOperator` with as many codomain as
    domain variables; ``grid``: the global grid; ``degree``: DG degree of every field. Rank and
    size come from the default process group (or ``group``); without an initialised process
    group the grid is one part."""

    def __init__(self, op, grid, degree, device=None, group=None, kernel=C.KERNEL_AUTO):
        import torch
        import torch.distributed as dist
        if not isinstance(grid, CartesianGrid):
            raise TypeError("grid must be a CartesianGrid")
        if dist.is_available() and dist.is_initialized():
            nranks, rank = dist.get_world_size(group), dist.get_rank(group)
        else:
            nranks, rank = 1, 0
        nvar = len(op.DomainVar)
        if len(op.CodomainVar) != nvar:
            raise ValueError("partitioned evaluation needs as many codomain as domain variables")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.part = SlabPartition(grid, nranks, rank, nvar * np_of(grid.dim, degree))
        self.halo = HaloExchange(self.part, group)
        self.ev = PartEvaluator(op, grid, [degree] * nvar, [degree] * nvar, self.part, self.device.index, kernel)
        self.time = 0.0

    def Dispose(self):
        self.ev.Dispose()

    def new_vector(self):
        import torch
        return torch.zeros(self.part.n_dofs, dtype=torch.float64, device=self.device)

    def own(self, x):
        return self.part.own(x)

    def _run(self, mode, U, V, out, alpha, beta, exchange):
        vecs = (U,) if V is None else (U, V)
        reqs = self.halo.start(*vecs) if exchange else []
        self.ev.apply(mode, U, V, out, self.part.interior_cells(), alpha, beta, self.time)
        HaloExchange.wait(reqs)
        for cells in self.part.rim_cells():
            self.ev.apply(mode, U, V, out, cells, alpha, beta, self.time)
        return out

    def Evaluate(self, alpha, beta, out, U, exchange=True):
        """``own(out) = beta*own(out) + alpha*Op(U)`` on the owned cells; U, out: part vectors
        whose owned DOFs are set (the exchange fills the ghost planes of U)."""
        return self._run(C.MODE_RESIDUAL, U, None, out, alpha, beta, exchange)

    def jvp(self, U, V, out, exchange=True):
        """J(U) V on the owned cells (ghost planes of U and V exchanged)."""
        return self._run(C.MODE_JVP, U, V, out, 1.0, 0.0, exchange)

    def vjp(self, U, W, out, exchange=True):
        """J(U)^T W on the owned cells (ghost planes of U and W exchanged)."""
        return self._run(C.MODE_VJP, U, W, out, 1.0, 0.0, exchange)
