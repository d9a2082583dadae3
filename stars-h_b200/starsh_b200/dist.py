"""One TLR matrix split over processes (one per GPU) with torch.distributed:
NCCL between the GPUs of a node, gloo on CPU.

This is the layer the reference's MPI backend provides
(src/backends/mpi/blrm/{drsdd,dmml,dfe}.c), over this library's C ABI:

* the blocks of the TLR format are dealt to the ranks by block rows:
  contiguous ranges of block rows, balanced by matrix entries (the
  reference deals them 2-D block-cyclically, src/control/blrf.c:577-715;
  whole block rows keep every output row of a product on one rank);
* every rank approximates its own blocks on its own GPU (no exchange: the
  points are replicated, every block is independent);
* the product B = M A broadcasts A from the root and sums the ranks'
  partial products onto the root, as the reference does
  (src/backends/mpi/blrm/dmml.c:60 MPI_Bcast, :212 MPI_Reduce);
* the error sums sum ||D - U V^T||^2 and sum ||D||^2 over the ranks'
  blocks with one all-reduce of two doubles
  (src/backends/mpi/blrm/dfe.c:146 MPI_Allreduce).

The compute goes through a backend object (B200Backend below: this
library on the rank's GPU), so the same partition and collectives run with
any implementation of the four operations.
"""
import ctypes
import math
from ctypes import POINTER, byref, c_double

import numpy as np


def split_block_rows(row_sizes, world):
    """Contiguous ranges [lo, hi) of block rows, one per rank, with about
    equal sums of row sizes (every block row spans all columns, so its
    entries are proportional to its size)."""
    sizes = np.asarray(row_sizes, dtype=np.float64)
    nb = len(sizes)
    if world <= 0:
        raise ValueError("world must be positive")
    cum = np.concatenate([[0.0], np.cumsum(sizes)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        # first block row whose start reaches r / world of the entries
        b = int(np.searchsorted(cum, total * r / world, side="left"))
        bounds.append(min(max(b, bounds[-1]), nb))
    bounds.append(nb)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def local_blocks(block_far, block_near, lo, hi):
    """Indices of the far and near blocks whose block row is in [lo, hi)
    (block lists as (n, 2) arrays of (row, column))."""
    far = np.asarray(block_far, dtype=np.int64).reshape(-1, 2)
    near = np.asarray(block_near, dtype=np.int64).reshape(-1, 2)
    fi = np.nonzero((far[:, 0] >= lo) & (far[:, 0] < hi))[0] if len(far) else far[:0, 0]
    ni = np.nonzero((near[:, 0] >= lo) & (near[:, 0] < hi))[0] if len(near) else near[:0, 0]
    return fi, ni


class Shard:
    """A rank's part of the matrix: its format and approximation."""

    def __init__(self, M, F, lo, hi):
        self.M, self.F, self.lo, self.hi = M, F, lo, hi


def _collective_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def approximate_sharded(backend, F, maxrank, tol, rank, world, engine=1):
    """The rank's blocks of format F (any STARSH_blrf pointer of the
    backend's library) approximated by the backend; returns a Shard."""
    Fc = F.contents
    R = Fc.row_cluster.contents
    sizes = [R.size[i] for i in range(Fc.nbrows)]
    lo, hi = split_block_rows(sizes, world)[rank]
    nf, nn = Fc.nblocks_far, Fc.nblocks_near
    far = np.ctypeslib.as_array(Fc.block_far, shape=(2 * nf,)).copy() if nf else np.zeros(0, np.int64)
    near = np.ctypeslib.as_array(Fc.block_near, shape=(2 * nn,)).copy() if nn else np.zeros(0, np.int64)
    fi, ni = local_blocks(far, near, lo, hi)
    Fl = backend.sub_format(F, far.reshape(-1, 2)[fi], near.reshape(-1, 2)[ni])
    M = backend.approximate(Fl, maxrank, tol, engine)
    return Shard(M, Fl, lo, hi)


def dmml_sharded(backend, shard, A, root=0):
    """B = M A over the ranks: A (N x nrhs, column-major, float64) is taken
    from the root and broadcast; every rank multiplies its blocks; the
    partial products are summed onto the root, which gets B (the other
    ranks get None)."""
    import torch
    import torch.distributed as dist
    dev = _collective_device()
    t = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)   # nrhs x N
    dist.broadcast(t, src=root)
    A_local = np.asfortranarray(t.cpu().numpy().T)
    B = backend.dmml(shard.M, A_local)
    tb = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
    dist.reduce(tb, dst=root, op=dist.ReduceOp.SUM)
    if dist.get_rank() != root:
        return None
    return np.asfortranarray(tb.cpu().numpy().T)


def dfe_sharded(backend, shard):
    """sqrt(sum diff2 / sum norm2) over the ranks' blocks (every rank gets
    the value)."""
    import torch
    import torch.distributed as dist
    diff2, norm2 = backend.dfe_sums(shard.M)
    t = torch.tensor([diff2, norm2], dtype=torch.float64,
                     device=_collective_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    d, n = float(t[0]), float(t[1])
    return math.sqrt(d) / math.sqrt(n) if n > 0 else 0.0


class B200Backend:
    """The four operations with this library on the calling rank's GPU."""

    def __init__(self, lib):
        self.lib = lib

    def sub_format(self, F, far_pairs, near_pairs):
        import starsh_b200 as sb
        Fc = F.contents
        nf, nn = len(far_pairs), len(near_pairs)
        libc = ctypes.CDLL("libc.so.6")
        libc.malloc.restype = ctypes.c_void_p

        def owned(pairs):
            # the new format takes ownership of malloc'd block lists
            if len(pairs) == 0:
                return None
            p = libc.malloc(ctypes.c_size_t(16 * len(pairs)))
            arr = (sb.STARSH_int * (2 * len(pairs))).from_address(p)
            arr[:] = [int(x) for x in np.asarray(pairs).ravel()]
            return ctypes.cast(p, POINTER(sb.STARSH_int))

        Fl = POINTER(sb.Blrf)()
        fn = self.lib.starsh_blrf_new_from_coo
        fn.restype = ctypes.c_int
        info = fn(byref(Fl), Fc.problem, Fc.symm, Fc.row_cluster,
                  Fc.col_cluster, sb.STARSH_int(nf), owned(far_pairs),
                  sb.STARSH_int(nn), owned(near_pairs), ctypes.c_int(1))
        if info != 0:
            raise RuntimeError(f"starsh_blrf_new_from_coo: {info}")
        return Fl

    def approximate(self, F, maxrank, tol, engine):
        import starsh_b200 as sb
        M = POINTER(sb.Blrm)()
        info = self.lib.starsh_b200_approximate(byref(M), F, maxrank, tol, 0,
                                                engine, 0)
        if info != 0:
            raise RuntimeError(self.lib.starsh_b200_last_error())
        return M

    def dmml(self, M, A):
        n, nrhs = A.shape
        B = np.zeros((n, nrhs), order="F")
        A = np.asfortranarray(A, dtype=np.float64)
        info = self.lib.starsh_blrm__dmml_b200(
            M, nrhs, 1.0, A.ctypes.data_as(POINTER(c_double)), n, 0.0,
            B.ctypes.data_as(POINTER(c_double)), n)
        if info != 0:
            raise RuntimeError(self.lib.starsh_b200_last_error())
        return B

    def dfe_sums(self, M):
        d, n = c_double(), c_double()
        if self.lib.starsh_b200_blrm_dfe_sums(M, byref(d), byref(n)) != 0:
            raise RuntimeError(self.lib.starsh_b200_last_error())
        return d.value, n.value

    def free(self, shard):
        self.lib.starsh_blrm_free(shard.M)
        self.lib.starsh_blrf_free(shard.F)
