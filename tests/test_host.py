"""Host-side logic of the FLOW mirror that needs no GPU: the reference's step
schedule, the .bin reader and the flow/confNNNN.dat writer."""
import json
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

from latticeyangmills_b200 import WilsonFlow, get_input_list, read_conf, write_conf, write_flow_obs


@pytest.mark.parametrize("tau,eps,rows", [(1.0, 0.01, 100), (4.0, 0.01, 400), (2.0, 0.01, 200),
                                          (0.05, 0.01, 5), (6.0, 0.02, 300), (0.3, 0.1, 2)])
def test_row_count_follows_reference(tau, eps, rows):
    # int(tauFinal/epsilon) rows, row 0 at t = 0 (src/Apps/wilsonflow.cpp:117)
    assert WilsonFlow(tau, eps).nrows() == rows == int(tau / eps)


def test_flow_file_format(tmp_path):
    m = [[0.0, 0.5, -0.25, -123.456789], [0.01, 0.6, 1e-7, -1.0]]
    p = write_flow_obs(tmp_path, 3, m)
    assert p.name == "conf0003.dat" and p.parent.name == "flow"
    text = p.read_text()
    # header and "%lf\t" cells of src/InputOutput/outputobs.cpp:66-81
    assert text == ("Flow Time\tPlaq.\tTopc.\tEnerg.\t\n"
                    "0.000000\t0.500000\t-0.250000\t-123.456789\t\n"
                    "0.010000\t0.600000\t0.000000\t-1.000000\t\n")


def test_read_conf_layout_and_size_check(tmp_path):
    n = (2, 3, 4, 5)
    a = np.arange(np.prod(n) * 72, dtype=np.float64)
    write_conf(tmp_path / "c.bin", a)
    U = read_conf(tmp_path / "c.bin", n)
    assert U.shape == (5, 4, 3, 2, 4, 18)
    # element k of link mu at (x,y,z,t) sits at ((site*4 + mu)*18 + k)
    x, y, z, t, mu, k = 1, 2, 3, 4, 2, 7
    site = x + 2 * (y + 3 * (z + 4 * t))
    assert U[t, z, y, x, mu, k] == (site * 4 + mu) * 18 + k
    with pytest.raises(ValueError):
        read_conf(tmp_path / "c.bin", (2, 3, 4, 4))


def test_input_list_sorted_bin_only(tmp_path):
    for name in ["conf0002.bin", "conf0000.bin", "notes.txt", "conf0001.bin"]:
        (tmp_path / name).write_bytes(b"")
    assert [p.split("/")[-1] for p in get_input_list(tmp_path)] == ["conf0000.bin", "conf0001.bin", "conf0002.bin"]


APP = ROOT / "latticeyangmills_b200" / "bin" / "ymflow_flow"


def _app_input(tmp_path, extra):
    indir = tmp_path / "in"
    indir.mkdir()
    shutil.copy(GOLDEN / "g4_expiah.bin", indir / "conf0000.bin")
    text = (GOLDEN / "app_flow" / "input.json").read_text()
    cfg = json.loads(text.replace("@IN@", str(indir)).replace("@OUT@", str(tmp_path / "out")))
    cfg.update(extra)
    (tmp_path / "run.json").write_text(json.dumps(cfg))
    return tmp_path / "run.json"


PGFG_OK = {"startType": "Cold", "MCSteps": 6, "thermSteps": 4, "SU3eps": 0.24, "NConf": 3}


@pytest.mark.parametrize("bad,msg", [
    ({"App": {"type": "FLOW", "params": {"epsilon": 0.01}}}, "wrong \"FLOW\" app specification"),
    ({"App": {"type": "PGFG", "params": {}}}, "wrong \"PGFG\" app specification"),
    ({"App": {"type": "PGFG", "params": dict(PGFG_OK, NCorr=2)}}, "wrong \"PGFG\" app specification"),
    ({"App": {"type": "PGFG", "params": dict(PGFG_OK, startType="Warm")}}, "startType must be"),
    ({"App": {"type": "PGFG", "params": dict(PGFG_OK, NConf=7)}}, "need 1 <= NConf <= MCSteps"),
    ({"App": {"type": "PGFG", "params": {k: v for k, v in dict(PGFG_OK, NCorr=0).items() if k != "NConf"}}},
     "NCorr must be >= 1"),
    ({"App": {"type": "PGFG", "params": dict(PGFG_OK, SU3eps=1.5)}}, "SU3eps must lie in (0, 1)"),
    ({"App": {"type": "PGFG", "params": PGFG_OK}, "MetropolisHits": 0}, "MetropolisHits must be >= 1"),
    ({"App": {"type": "GFR", "params": {}}}, "\"FLOW\" and \"PGFG\" are provided"),
    ({"Observables": ["wilsonloop"]}, "unknown Observable"),
    ({"LatticeSize": {"x": 4, "y": 4, "z": 4}}, "wrong LatticeSize specification"),
    ({"Precision": "fp16"}, "unknown Precision"),
    ({"Endian": "middle"}, "unknown Endian"),
    ({"IOChunkSites": 0}, "IOChunkSites must be >= 1"),
])
def test_flow_app_rejects_bad_input(tmp_path, bad, msg):
    # validation as the reference's JsonInput layer, before any device work
    run = _app_input(tmp_path, bad)
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True)
    assert res.returncode == 1 and msg in res.stderr


def test_big_endian_conf_round_trip(tmp_path):
    from latticeyangmills_b200 import read_conf, write_conf

    n = (4, 4, 4, 4)
    U = read_conf(GOLDEN / "g4_expiah.bin", n)
    write_conf(tmp_path / "be.bin", U, big_endian=True)
    raw = (tmp_path / "be.bin").read_bytes()
    assert raw[:8] == U.reshape(-1)[:1].astype(">f8").tobytes()
    assert raw != (GOLDEN / "g4_expiah.bin").read_bytes()
    assert np.array_equal(read_conf(tmp_path / "be.bin", n, big_endian=True), U)


def test_slab_partition_tiles_the_time_extent():
    from latticeyangmills_b200 import slab_partition

    for nt_global in (1, 7, 32, 33):
        for nranks in range(1, min(nt_global, 9) + 1):
            parts = [slab_partition(nt_global, nranks, r) for r in range(nranks)]
            assert parts[0][0] == 0
            assert sum(p[1] for p in parts) == nt_global
            assert max(p[1] for p in parts) - min(p[1] for p in parts) <= 1
            for r, (t0, nt, lo, hi) in enumerate(parts):
                if r + 1 < nranks:
                    assert parts[r + 1][0] == t0 + nt
                assert parts[lo][0] + parts[lo][1] == t0 or (r == 0 and lo == nranks - 1)
                assert parts[hi][2] == r
    with pytest.raises(ValueError):
        slab_partition(4, 5, 0)


REF_GPU_APP = ROOT / "oracle" / "_ref" / "lattice_qcd_ymflow"


@pytest.mark.skipif(not REF_GPU_APP.exists(), reason="oracle/_ref/lattice_qcd_ymflow not built (no reference tree)")
def test_reference_registry_reaches_the_gpu_wilsonflow(tmp_path):
    """The reference's JSON layer builds its FLOW app from the adapter's
    WilsonFlow: without a B200 the adapter's device set-up is what stops it."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: tests/test_gpu_app.py runs the application")
    run = _app_input(tmp_path, {})
    res = subprocess.run([str(REF_GPU_APP), str(run)], capture_output=True, text=True)
    assert res.returncode == 1
    assert "ymflow create" in res.stderr


def test_bench_byte_accounting_and_profiled_traffic():
    """The roofline numerators of bench.py: the fused stage's compulsory bytes
    per link-update, the two-kernel stage's per kernel, and the DRAM traffic
    scaled from the committed ncu summaries."""
    import bench

    assert [bench.bytes_per_link_update(p) for p in ("fp64", "fp32_18", "fp32_12")] == [1120, 560, 416]
    field, stage = bench.split_bytes_per_link("fp32_12")
    assert field == 96 and stage == pytest.approx(186.6667, rel=1e-5)
    assert 3 * (field + stage) == pytest.approx(848)
    field, stage = bench.split_bytes_per_link("fp32_18")
    assert field == 120 and 3 * (field + stage) == pytest.approx(1064)
    alg = 1e9
    got = bench.profiled_traffic("fp32_12", (32, 32, 32, 32), alg, "rk_split_stage")
    assert got == pytest.approx(846300928 / 671088640 * alg)
    got = bench.profiled_traffic("fp32_12", (32, 32, 32, 32), alg, "plaq_field")
    assert got == pytest.approx(369448704 / 402653184 * alg)
    got = bench.profiled_traffic("fp64", (32, 32, 32, 32), alg, "rk_stage")
    assert got == pytest.approx(1860280032 / 1744830464 * alg)
    assert bench.profiled_traffic("fp32_12", (16, 16, 16, 16), alg, "rk_split_stage") is None


def test_bench_roofline_on_compulsory_bytes():
    """bench.py's HBM fractions on the compulsory bytes of the three stages
    (416 B per link-update for FP32-12): one stage launch carries a third of
    them; the step fraction is link-updates/s x bytes.  The numbers of the
    first measured line (0.2029 ms per stage launch, 4.27e9 LU/s) give the
    kernel and step fractions 0.44 and 0.27 of 6549 GB/s."""
    import bench

    links = 4 * 32 ** 4
    r = bench.roofline_8d("fp32_12", links, 4.27e9, 0.2029e-3, 6549.0)
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(416 / 3 * links)
    assert r["achieved"] == pytest.approx(416 / 3 * links / 0.2029e-3 / 1e9)
    assert r["frac"] == pytest.approx(0.4377, abs=5e-4)
    assert r["step_achieved"] == pytest.approx(4.27e9 * 416 / 1e9)
    assert r["step_frac"] == pytest.approx(0.2712, abs=5e-4)
    r64 = bench.roofline_8d("fp64", links, 2.11e9, 0.5e-3, 6549.0)
    assert r64["step_frac"] == pytest.approx(2.11e9 * 1120 / 1e9 / 6549.0)
