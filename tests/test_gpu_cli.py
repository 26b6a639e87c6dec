"""End-to-end runs of the command line on the GPU: a seeded synthetic cohort written as
PLINK BED, single K with Adam-EM and a K sweep with SQP + ZAL and cross-validation. Checks
the files (reference text format, feasibility), that the CLI's result equals the Python
API's on the same inputs, and that the fit recovers the simulated ancestry."""
import numpy as np
import pytest
import torch

from adamixture_b200.src.align import align_clusters
from adamixture_b200.src.simulate import make_cohort, write_bed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort(tmp_path_factory, cuda):
    d = tmp_path_factory.mktemp("cohort")
    coh = make_cohort(300, 4000, 3, F=0.1, alpha=0.5, miss=0.01, seed=12)
    write_bed(d / "sim", coh.genotypes())
    return d, coh


def run(args):
    from adamixture_b200 import cli

    assert cli.main(args) == 0


def test_single_k_adamem(cohort, tmp_path):
    d, coh = cohort
    run(["--k", "3", "--data_path", str(d / "sim.bed"), "--save_dir", str(tmp_path), "--name", "a",
         "--algorithm", "adamem", "--precision", "f64"])
    Q = np.loadtxt(tmp_path / "a.3.Q")
    P = np.loadtxt(tmp_path / "a.3.P")
    assert Q.shape == (300, 3) and P.shape == (4000, 3)
    np.testing.assert_allclose(Q.sum(1), 1.0, atol=1e-9)
    assert P.min() >= 1e-5 - 1e-15 and P.max() <= 1 - 1e-5 + 1e-15
    perm = align_clusters(coh.Q, Q)
    assert np.abs(Q[:, perm] - coh.Q).mean() < 0.03
    # the CLI equals the Python API on the same inputs
    from adamixture_b200.src import utils
    from adamixture_b200.src.adamixture import setup, train_k

    G, N, M = utils.read_data(str(d / "sim.bed"), device=torch.device("cuda"))
    dev, tpb, f, U, S, V, G = setup(G, N, M, 3, 42, 5, 0.1, 8192, "gpu")
    P2, Q2 = train_k(G, N, M, 3, U, S, V, f, 42, 0.005, 0.8, 0.88, 1e-8, 10000, 5, 1000, 1e-4, 0.5, 1e-4,
                     8192, 3, 0.1, dev, tpb, precision="f64")
    np.testing.assert_allclose(Q, Q2.cpu().numpy(), atol=1e-15)


def test_sweep_brqn_with_cv(cohort, tmp_path):
    d, coh = cohort
    run(["--min_k", "2", "--max_k", "4", "--data_path", str(d / "sim.bed"), "--save_dir", str(tmp_path),
         "--name", "b", "--cv", "3", "--no_freqs"])
    for K in (2, 3, 4):
        Q = np.loadtxt(tmp_path / f"b.{K}.Q")
        assert Q.shape == (300, K)
        np.testing.assert_allclose(Q.sum(1), 1.0, atol=1e-9)
        assert not (tmp_path / f"b.{K}.P").exists()
    Q3 = np.loadtxt(tmp_path / "b.3.Q")
    perm = align_clusters(coh.Q, Q3)
    assert np.abs(Q3[:, perm] - coh.Q).mean() < 0.03


def test_bed_decode_leaves_the_estep_status_word_alone(cuda, synth):
    # the on-device BED decode runs between E-steps in a real run; its scratch must not be
    # the E-step workspace whose first word is the sweep's status
    from adamixture_b200 import ops

    M, N, K = int(synth["M"]), int(synth["N"]), int(synth["K"])
    G = torch.from_numpy(synth["packed"]).cuda()
    P = torch.from_numpy(synth["P0"]).cuda().float()
    Q = torch.from_numpy(synth["Q0"]).cuda().float()
    ops.em_stats(G, P, Q, M, "bf16")
    ws = ops.Workspace.get(G.device, ops.em_workspace_bytes(M, N, K, "bf16"))
    rng = np.random.default_rng(0)
    rows = torch.from_numpy(rng.integers(0, 256, size=(M, (N + 3) // 4), dtype=np.uint8)).cuda()
    ops.bed_to_packed(rows, N, M)
    assert ops.em_status(ws, M, N, K, "bf16") == 0
