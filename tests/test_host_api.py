"""Host-side mirror of the reference interface (no GPU)."""
import json

import numpy as np

from distributed_diskann_b200 import datasets as D
from distributed_diskann_b200.index import DatasetPara, Graph, PointRange


def test_dataset_para_reads_reference_json(tmp_path):
    para = {"build": True, "save": True, "query": False, "two_pass": False,
            "data_para": str(tmp_path / "ds.json"), "start_point_index": 0, "xita": 1,
            "alpha": 1.2, "L": 64, "R": 32, "Ls": 100, "num_neighbors_query": 10, "max": 0}
    ds = {"dataset": "random-xs", "nb": 10000, "nq": 1000, "d": 20, "dtype": "float32",
          "ds_fn": "data_10000_20", "qs_fn": "queries_1000_20", "gt_fn": "gt_10000_1000_20",
          "basedir": "data/random10000"}
    (tmp_path / "para.json").write_text(json.dumps(para))
    (tmp_path / "ds.json").write_text(json.dumps(ds))
    dp = DatasetPara()
    dp.set(str(tmp_path / "para.json"))
    dp.open(dp.dataset_parafile)
    assert (dp.R, dp.L, dp.alpha, dp.xita, dp.max_build) == (32, 64, 1.2, 1, 0)
    assert dp.ds_dir == "data/random10000/data_10000_20"
    assert dp.output_path == "results/random-xs"


def test_graph_file_roundtrip_matches_oracle_format(tmp_path, oracle_mod):
    rng = np.random.default_rng(0)
    n, R = 50, 6
    g = Graph(R, n)
    deg = rng.integers(0, R + 1, n)
    for i in range(n):
        g.rows[i, 0] = deg[i]
        g.rows[i, 1 : 1 + deg[i]] = rng.integers(0, n, deg[i])
    g.save(str(tmp_path / "g.bin"))
    g2 = Graph(path=str(tmp_path / "g.bin"))
    np.testing.assert_array_equal(g.rows, g2.rows)
    np.testing.assert_array_equal(oracle_mod.read_graph(str(tmp_path / "g.bin")), g.rows)


def test_bin_roundtrip(tmp_path):
    x = np.arange(60, dtype=np.int8).reshape(6, 10)
    D.write_bin(str(tmp_path / "x.bin"), x)
    np.testing.assert_array_equal(PointRange(str(tmp_path / "x.bin"), np.int8).values, x)


def test_recall_with_ties():
    gt_i = np.array([[1, 2, 3, 4]])
    gt_d = np.array([[0.0, 1.0, 2.0, 2.0]], np.float32)
    # k = 3: the tie at the 3rd distance admits id 4 too
    assert D.recall_with_ties(np.array([[1, 2, 4]]), gt_i, gt_d, 3) == 1.0
