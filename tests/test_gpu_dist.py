"""The split layer (starsh_b200.dist) with this library as the backend, on
one GPU as a one-rank group: the sharded product equals the library's
product of the whole matrix and the all-reduced error sums give its dfe.
(Several ranks need several GPUs; the partition and collectives are
checked with two gloo ranks in test_dist.py.)"""
import ctypes
import os
import socket
from ctypes import POINTER, byref, c_double

import numpy as np
import pytest

import oracle
import starsh_b200 as sb
from harness import RefProblem, approximate_b200, as_ref_blrm


@pytest.mark.gpu
def test_one_rank_split_matches_whole_matrix(ref, lib):
    import torch.distributed as dist
    from starsh_b200 import dist as sd
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}",
                            rank=0, world_size=1)
    try:
        be = sd.B200Backend(lib)
        pr = RefProblem(ref, "spatial", 3600, 400, kernel_name="exp", beta=0.1)
        lib.starsh_set_oversample(b"10")
        shard = sd.approximate_sharded(be, pr.b200_format(), 100, 1e-5, 0, 1,
                                       engine=sb.ENGINE_MIXED)
        A = np.asfortranarray(np.random.default_rng(2).standard_normal((3600, 4)))
        B = sd.dmml_sharded(be, shard, A)
        err = sd.dfe_sharded(be, shard)
        assert err == pytest.approx(lib.starsh_blrm__dfe_b200(shard.M), rel=1e-12)
        assert 0 < err <= 1e-5
        d, n = c_double(), c_double()
        assert lib.starsh_b200_blrm_dfe_sums(shard.M, byref(d), byref(n)) == 0
        assert np.sqrt(d.value / n.value) == pytest.approx(err, rel=1e-14)
        # the product against the same approximation multiplied whole
        lib.starsh_b200_blrm_download(shard.M)
        Bw = ref.dmml(as_ref_blrm(shard.M), A)
        assert np.max(np.abs(B - Bw)) <= 1e-12 * np.max(np.abs(Bw))
        be.free(shard)
    finally:
        dist.destroy_process_group()
