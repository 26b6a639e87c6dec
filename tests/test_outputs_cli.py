"""Host-side pieces of the run driver: the native .Q/.P writer (byte-identical to the
reference's np.savetxt), cluster alignment across K (against the reference's own
alignment, tests/golden/align.npz) and the command line."""
import numpy as np
import pytest

from adamixture_b200 import cli, project_entry, supervised_entry
from adamixture_b200.src import align, utils


def test_writer_is_byte_identical_to_savetxt(tmp_path):
    rng = np.random.default_rng(3)
    Q = rng.dirichlet(np.ones(5), 9001)
    P = rng.uniform(1e-5, 1 - 1e-5, (777, 5))
    P[0, 0], P[1, 1], P[2, 2] = 0.0, -0.0, 1e-300
    utils.write_outputs(Q, "run", 5, tmp_path, P=P)
    np.savetxt(tmp_path / "q.ref", Q, delimiter=" ")
    np.savetxt(tmp_path / "p.ref", P, delimiter=" ")
    assert (tmp_path / "run.5.Q").read_bytes() == (tmp_path / "q.ref").read_bytes()
    assert (tmp_path / "run.5.P").read_bytes() == (tmp_path / "p.ref").read_bytes()
    utils.write_outputs(Q[:, :1].ravel(), "one", 1, tmp_path)
    assert not (tmp_path / "one.1.P").exists()
    np.testing.assert_array_equal(np.loadtxt(tmp_path / "one.1.Q"), Q[:, 0])


def test_fixed_writer_is_byte_identical_to_savetxt(tmp_path):
    """"%.6f" as the projection and supervised commands write (np.savetxt fmt="%.6f"),
    including exact decimal ties (k / 2**7 has 7 decimals), signed zeros, large values and
    non-finite values."""
    rng = np.random.default_rng(5)
    Q = rng.dirichlet(np.ones(4), 5000)
    P = rng.uniform(1e-5, 1 - 1e-5, (4099, 4))
    P[:128, 0] = np.arange(128) / 128.0
    P[:128, 1] = -np.arange(128) / 128.0
    P[128:136, 2] = [0.0, -0.0, -1e-9, 1e300, -2.5e17, np.inf, -np.inf, np.nan]
    P[136:, 3] = np.round(P[136:, 3], 7) + 5e-7
    utils.write_outputs(Q, "f", 4, tmp_path, P=P, decimals=6)
    np.savetxt(tmp_path / "q.ref", Q, delimiter=" ", fmt="%.6f")
    np.savetxt(tmp_path / "p.ref", P, delimiter=" ", fmt="%.6f")
    assert (tmp_path / "f.4.Q").read_bytes() == (tmp_path / "q.ref").read_bytes()
    assert (tmp_path / "f.4.P").read_bytes() == (tmp_path / "p.ref").read_bytes()
    utils.write_outputs(Q, "g", 4, tmp_path, decimals=0)
    np.savetxt(tmp_path / "g.ref", Q, delimiter=" ", fmt="%.0f")
    assert (tmp_path / "g.4.Q").read_bytes() == (tmp_path / "g.ref").read_bytes()


def test_project_command_options():
    a = project_entry.parse_args(["--data_path", "t.bed", "--p_path", "r.4.P", "--save_dir", "o",
                                  "--name", "n", "--algorithm", "adamem", "--seed", "3"])
    assert (a.algorithm, a.seed, a.chunk_size, a.max_iter, a.check, a.device) == ("adamem", 3, 4096, 10000, 5, "cuda")
    for bad in (["--lr", "0"], ["--beta1", "1"], ["--lr_decay", "0"], ["--check", "0"], ["--device", "cpu"]):
        with pytest.raises(SystemExit):
            project_entry.parse_args(["--data_path", "t", "--p_path", "p", "--save_dir", "o", "--name", "n", *bad])
    with pytest.raises(SystemExit):
        project_entry.parse_args(["--data_path", "t", "--save_dir", "o", "--name", "n"])


def test_supervised_command_options_and_labels(tmp_path):
    base = ["--data_path", "t.bed", "--save_dir", "o", "--name", "n", "--labels", "l1.txt"]
    a = supervised_entry.parse_args(base + ["--no_freqs"])
    assert (a.level, a.no_freqs, a.algorithm) == (1, True, "brqn")
    for bad in (["--k", "3"], ["--min_k", "2"], ["--level", "2"], ["--level", "4"]):
        with pytest.raises(SystemExit):
            supervised_entry.parse_args(base + bad)
    assert supervised_entry.parse_args(base + ["--level", "2", "--labels2", "l2.txt"]).labels2 == "l2.txt"
    f = tmp_path / "labels.txt"
    f.write_text("-\nYRI\n\n CEU \nYRI\n-\nCHB\nCEU\n")
    raw = supervised_entry.parse_labels_file(f)
    assert raw == ["-", "YRI", "CEU", "YRI", "-", "CHB", "CEU"]
    y, names = supervised_entry.labels_to_y(raw)
    assert y.dtype == np.int32 and y.tolist() == [0, 1, 2, 1, 0, 3, 2]
    assert names == {"YRI": 1, "CEU": 2, "CHB": 3}


@pytest.mark.parametrize("c", range(6))
def test_alignment_matches_reference(align_golden, c):
    d = align_golden
    np.testing.assert_array_equal(align.align_clusters(d[f"c{c}_ref"], d[f"c{c}_query"]), d[f"c{c}_perm"])


def test_cli_parses_reference_options():
    a = cli.parse_args(["--min_k", "2", "--max_k", "4", "--data_path", "x.bed", "--save_dir", "o",
                        "--name", "n", "--algorithm", "adamem", "--cv", "--seed", "7"])
    assert (a.min_k, a.max_k, a.cv, a.seed, a.algorithm, a.device) == (2, 4, 5, 7, "adamem", "gpu")
    with pytest.raises(SystemExit):
        cli.parse_args(["--data_path", "x", "--save_dir", "o", "--name", "n"])
    with pytest.raises(SystemExit):
        cli.parse_args(["--k", "3", "--device", "cpu", "--data_path", "x", "--save_dir", "o", "--name", "n"])


def test_precision_policy():
    """auto: the FP16 tensor-core sweep for 8 <= K <= 16, float32 SIMT otherwise; the
    tensor-core forms take any K <= 16 on request and refuse K > 16."""
    from adamixture_b200.model.em_adam_gpu import resolve_precision

    assert [resolve_precision(K, "auto") for K in (1, 2, 7, 8, 10, 16, 17, 64)] == \
        ["f32", "f32", "f32", "f16", "f16", "f16", "f32", "f32"]
    assert resolve_precision(3, "f16") == "f16"
    assert resolve_precision(10, "mixed") == "f16" and resolve_precision(10, "bf16") == "bf16"
    for p in ("bf16", "f16"):
        with pytest.raises(ValueError):
            resolve_precision(17, p)
    assert resolve_precision(3, "f64") == "f64"
