"""The SNP-sharded Adam-EM on the GPU through a one-rank NCCL group: the CUDA backend's
separate statistics / all-reduce / targets / Adam path matches the fused single-GPU
optimiser in float64 (the collective is an identity on one rank; the multi-rank exchange
is covered by the two-rank gloo test on the CPU)."""
import socket

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("prec,atol,rel", [("f64", 1e-9, 1e-12), ("f16", 1e-6, 1e-9)])
def test_one_rank_sharded_matches_fused(cuda, synth, prec, atol, rel):
    # the sharded path (statistics, all-reduce, targets, Adam as separate launches) against
    # the fused optimiser: the same iterates and the same checks (the float32-h check for
    # the 16-bit sweep on both paths)
    import torch.distributed as dist

    from adamixture_b200.model.em_adam_dist import CudaBackend, optimize_parameters_dist
    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    G = torch.from_numpy(synth["packed"]).cuda()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1,
                            device_id=cuda)
    tr1, tr2 = [], []
    try:
        P1, Q1 = optimize_parameters_dist(G, torch.from_numpy(synth["P0"]).cuda(), torch.from_numpy(synth["Q0"]).cuda(),
                                          0.005, 0.80, 0.88, 1e-8, 40, 5, K, M, N, 0.5, 1e-4, 3, 0.1,
                                          backend=CudaBackend(prec), trace=tr1)
    finally:
        dist.destroy_process_group()
    P2, Q2 = optimize_parameters_gpu(G, torch.from_numpy(synth["P0"]).cuda(), torch.from_numpy(synth["Q0"]).cuda(),
                                     0.005, 0.80, 0.88, 1e-8, 40, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 256,
                                     precision=prec, trace=tr2)
    np.testing.assert_allclose(P1.cpu().numpy(), P2.cpu().numpy(), atol=atol)
    np.testing.assert_allclose(Q1.cpu().numpy(), Q2.cpu().numpy(), atol=atol)
    assert [i for i, _ in tr1] == [i for i, _, _ in tr2]
    for (_, L1), (_, L2, _) in zip(tr1, tr2):
        assert abs(L1 - L2) <= rel * abs(L2), (L1, L2)
