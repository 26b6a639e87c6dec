"""Host-side pieces of the run driver: the native .Q/.P writer (byte-identical to the
reference's np.savetxt), cluster alignment across K (against the reference's own
alignment, tests/golden/align.npz) and the command line."""
import numpy as np
import pytest

from adamixture_b200 import cli
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
