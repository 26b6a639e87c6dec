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


def test_one_rank_sharded_matches_fused(cuda, synth):
    import torch.distributed as dist

    from adamixture_b200.model.em_adam_dist import CudaBackend, optimize_parameters_dist
    from adamixture_b200.model.em_adam_gpu import optimize_parameters_gpu

    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    G = torch.from_numpy(synth["packed"]).cuda()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1,
                            device_id=cuda)
    try:
        P1, Q1 = optimize_parameters_dist(G, torch.from_numpy(synth["P0"]).cuda(), torch.from_numpy(synth["Q0"]).cuda(),
                                          0.005, 0.80, 0.88, 1e-8, 40, 5, K, M, N, 0.5, 1e-4, 3, 0.1,
                                          backend=CudaBackend("f64"))
    finally:
        dist.destroy_process_group()
    P2, Q2 = optimize_parameters_gpu(G, torch.from_numpy(synth["P0"]).cuda(), torch.from_numpy(synth["Q0"]).cuda(),
                                     0.005, 0.80, 0.88, 1e-8, 40, 5, K, M, N, 0.5, 1e-4, 3, 0.1, G.device, 8192, 256,
                                     precision="f64")
    np.testing.assert_allclose(P1.cpu().numpy(), P2.cpu().numpy(), atol=1e-9)
    np.testing.assert_allclose(Q1.cpu().numpy(), Q2.cpu().numpy(), atol=1e-9)
