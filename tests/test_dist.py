"""The multi-process split of one TLR matrix (starsh_b200.dist): block-row
partition, the root's broadcast and reduce of the product, the all-reduce
of the error sums.  Checked with two gloo ranks on the CPU, the compiled
reference library standing in for the GPU as the compute backend: the
sharded product and error equal those of the whole matrix approximated in
one process (every block is compressed the same way wherever it is)."""
import ctypes
import os
import socket
import sys
from ctypes import POINTER, byref, c_int

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

from starsh_b200.dist import local_blocks, split_block_rows   # noqa: E402


def test_split_block_rows_is_a_balanced_partition():
    sizes = [100] * 7 + [40, 10]
    for world in (1, 2, 3, 4, 9, 12):
        parts = split_block_rows(sizes, world)
        assert len(parts) == world
        assert parts[0][0] == 0 and parts[-1][1] == len(sizes)
        for (a, b), (c, d) in zip(parts, parts[1:]):
            assert b == c and a <= b
        if world <= len(sizes):
            loads = [sum(sizes[a:b]) for a, b in parts]
            assert max(loads) - min(loads) <= max(sizes)


def test_local_blocks_selects_block_rows():
    far = np.array([[0, 1], [1, 0], [2, 0], [2, 1], [3, 3]])
    near = np.array([[0, 0], [3, 2]])
    fi, ni = local_blocks(far, near, 1, 3)
    assert list(fi) == [1, 2, 3] and list(ni) == []
    fi, ni = local_blocks(far, near, 3, 4)
    assert list(fi) == [4] and list(ni) == [1]


class RefBackend:
    """The four operations of the split with the compiled reference."""

    def __init__(self, ref, pr):
        import oracle
        self.ref, self.pr, self.oracle = ref, pr, oracle
        fn = ref.lib.starsh_blrf_new_from_coo
        fn.restype = c_int
        fn.argtypes = [POINTER(POINTER(oracle.Blrf)), ctypes.c_void_p,
                       ctypes.c_char, POINTER(oracle.Cluster),
                       POINTER(oracle.Cluster), oracle.STARSH_int,
                       POINTER(oracle.STARSH_int), oracle.STARSH_int,
                       POINTER(oracle.STARSH_int), c_int]

    def sub_format(self, F, far_pairs, near_pairs):
        o = self.oracle
        libc = ctypes.CDLL("libc.so.6")
        libc.malloc.restype = ctypes.c_void_p

        def owned(pairs):
            if len(pairs) == 0:
                return None
            p = libc.malloc(ctypes.c_size_t(16 * len(pairs)))
            arr = (o.STARSH_int * (2 * len(pairs))).from_address(p)
            arr[:] = [int(x) for x in np.asarray(pairs).ravel()]
            return ctypes.cast(p, POINTER(o.STARSH_int))

        Fc = F.contents
        Fl = POINTER(o.Blrf)()
        assert self.ref.lib.starsh_blrf_new_from_coo(
            byref(Fl), Fc.problem, Fc.symm, Fc.row_cluster, Fc.col_cluster,
            len(far_pairs), owned(far_pairs), len(near_pairs),
            owned(near_pairs), 1) == 0
        return Fl

    def approximate(self, F, maxrank, tol, engine):
        return self.ref.approximate(F, maxrank, tol, oversample=10,
                                    sequential=True)

    def dmml(self, M, A):
        return self.ref.dmml(M, A)

    def dfe_sums(self, M):
        # the two sums of src/backends/sequential/blrm/dfe.c:16-134
        c = self.oracle.blrm_contents(M)
        diff2 = norm2 = 0.0
        for b, (i, j) in enumerate(c["far"]):
            D = self.pr.block(i, j)
            norm2 += float(np.sum(D * D))
            E = D - c["U"][b] @ c["V"][b].T
            diff2 += float(np.sum(E * E))
        for b, (i, j) in enumerate(c["near"]):
            norm2 += float(np.sum(c["D"][b] ** 2))
        return diff2, norm2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    for p in ("stars-h_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(ROOT, p))
    import torch.distributed as dist
    import oracle
    from harness import RefProblem
    from starsh_b200 import dist as sd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ref = oracle.Ref()
        pr = RefProblem(ref, "spatial", 1600, 200, kernel_name="exp", beta=0.1)
        be = RefBackend(ref, pr)
        maxrank, tol = 60, 1e-6
        shard = sd.approximate_sharded(be, pr.F, maxrank, tol, rank, world)
        A = (np.random.default_rng(5).standard_normal((1600, 3))
             if rank == 0 else np.zeros((1600, 3)))
        A = np.asfortranarray(A)
        B = sd.dmml_sharded(be, shard, A)
        err = sd.dfe_sharded(be, shard)
        if rank == 0:
            # the whole matrix in this process, the same way
            pw = RefProblem(ref, "spatial", 1600, 200, kernel_name="exp", beta=0.1)
            M = ref.approximate(pw.F, maxrank, tol, oversample=10, sequential=True)
            out["B"] = B.tolist()
            out["B_full"] = ref.dmml(M, A).tolist()
            out["err"] = err
            out["err_full"] = ref.dfe(M)
        out[f"rows{rank}"] = (shard.lo, shard.hi)
    finally:
        dist.destroy_process_group()


def test_sharded_product_and_error_equal_one_process():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res["rows0"][0] == 0 and res["rows0"][1] == res["rows1"][0]
    assert res["rows1"][1] == 8
    B, Bf = np.array(res["B"]), np.array(res["B_full"])
    assert np.max(np.abs(B - Bf)) <= 1e-12 * np.max(np.abs(Bf))
    assert res["err"] == pytest.approx(res["err_full"], rel=1e-10)
    assert res["err"] <= 1e-6
