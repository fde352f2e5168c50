"""The drop-in FLOW driver (latticeyangmills_b200/bin/ymflow_flow) against the
reference's own FLOW application: same JSON, same .bin inputs, and byte-identical
terminal lines and output files (tests/golden/app_flow, produced by the
reference binary)."""
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

APP = ROOT / "latticeyangmills_b200" / "bin" / "ymflow_flow"


def prepare(tmp_path, extra=None):
    import json

    indir = tmp_path / "in"
    indir.mkdir()
    shutil.copy(GOLDEN / "g4_expiah.bin", indir / "conf0000.bin")
    shutil.copy(GOLDEN / "g4b_expiah.bin", indir / "conf0001.bin")
    (indir / "notes.txt").write_text("ignored: not a .bin\n")
    text = (GOLDEN / "app_flow" / "input.json").read_text()
    text = text.replace("@IN@", str(indir)).replace("@OUT@", str(tmp_path / "out"))
    cfg = json.loads(text)
    cfg.update(extra or {})
    (tmp_path / "run.json").write_text(json.dumps(cfg))
    return tmp_path / "run.json"


def test_flow_app_output_matches_reference_app(tmp_path):
    run = prepare(tmp_path)
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    got = [l for l in res.stdout.splitlines(keepends=True) if not l.startswith("Total time taken")]
    exp = GOLDEN / "app_flow" / "expected"
    assert "".join(got) == (exp / "stdout.txt").read_text()
    for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (exp / f).read_bytes(), f
    assert (tmp_path / "out" / "flow" / "conf0000.full.dat").exists()


REF_GPU_APP = ROOT / "oracle" / "_ref" / "lattice_qcd_ymflow"


@pytest.mark.skipif(not REF_GPU_APP.exists(), reason="oracle/_ref/lattice_qcd_ymflow not built (no reference tree)")
def test_reference_application_with_gpu_wilsonflow(tmp_path):
    """The reference's own LatticeQCD program (its main, JSON layer and I/O)
    with its WilsonFlow replaced by the libymflow adapter
    (latticeyangmills_b200/adapter/wilsonflow_ymflow.cpp): the same terminal
    lines and files as the unmodified reference application."""
    run = prepare(tmp_path)
    res = subprocess.run([str(REF_GPU_APP), str(run)], capture_output=True, text=True, check=True)
    got = [l for l in res.stdout.splitlines(keepends=True) if not l.startswith("Total time taken")]
    exp = GOLDEN / "app_flow" / "expected"
    assert "".join(got) == (exp / "stdout.txt").read_text()
    for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (exp / f).read_bytes(), f


def test_flow_app_big_endian_streamed_input(tmp_path):
    """Byte-reversed ("Chroma") inputs read in ragged chunks give the same
    files as the native-endian run."""
    import numpy as np

    run = prepare(tmp_path, {"Endian": "big", "IOChunkSites": 97})
    for name in ["conf0000.bin", "conf0001.bin"]:
        f = tmp_path / "in" / name
        f.write_bytes(np.fromfile(f, dtype="<f8").astype(">f8").tobytes())
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    got = [l for l in res.stdout.splitlines(keepends=True) if not l.startswith("Total time taken")]
    exp = GOLDEN / "app_flow" / "expected"
    assert "".join(got) == (exp / "stdout.txt").read_text()
    for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (exp / f).read_bytes(), f


def test_flow_app_time_slabs_from_sublattice_size(tmp_path):
    """A SubLatticeSize that splits only t flows each configuration as time
    slabs (here two, on the GPUs present): the same files as the reference
    application, and its terminal lines apart from the processor count."""
    run = prepare(tmp_path, {"SubLatticeSize": {"x": 4, "y": 4, "z": 4, "t": 2}})
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    got = [l for l in res.stdout.splitlines(keepends=True) if not l.startswith("Total time taken")]
    exp = (GOLDEN / "app_flow" / "expected" / "stdout.txt").read_text().splitlines(keepends=True)
    assert "Number of Processors: \t\t2\n" in got and "Number of Active Processors: \t2\n" in got
    keep = lambda lines: [l for l in lines if not l.startswith(("Number of", "Sublattice Size"))]
    assert keep(got) == keep(exp)
    ex = GOLDEN / "app_flow" / "expected"
    for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (ex / f).read_bytes(), f


@pytest.mark.parametrize("sub,nblocks", [({"x": 2, "y": 4, "z": 2, "t": 2}, 8), ({"x": 4, "y": 2, "z": 4, "t": 4}, 2),
                                         ({"x": 2, "y": 2, "z": 2, "t": 2}, 16)])
def test_flow_app_blocks_from_sublattice_size(tmp_path, sub, nblocks):
    """A SubLatticeSize that splits x, y or z flows each configuration as blocks
    in the reference's Cartesian layout (parallel.cpp:57-100): the same files as
    the reference application, its terminal lines apart from the processor
    count."""
    run = prepare(tmp_path, {"SubLatticeSize": sub})
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    got = [l for l in res.stdout.splitlines(keepends=True) if not l.startswith("Total time taken")]
    exp = (GOLDEN / "app_flow" / "expected" / "stdout.txt").read_text().splitlines(keepends=True)
    assert "Number of Processors: \t\t%d\n" % nblocks in got
    keep = lambda lines: [l for l in lines if not l.startswith(("Number of", "Sublattice Size"))]
    assert keep(got) == keep(exp)
    ex = GOLDEN / "app_flow" / "expected"
    for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (ex / f).read_bytes(), f


def test_flow_app_empty_input_dir(tmp_path):
    """No .bin files: the reference writes its headers and flows nothing."""
    run = prepare(tmp_path)
    for f in (tmp_path / "in").glob("*.bin"):
        f.unlink()
    res = subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    assert "Configuration Number" not in res.stdout
    assert (tmp_path / "out" / "observables.dat").read_text() == "Step\tSuperObs\t\n"
    assert not list((tmp_path / "out" / "flow").glob("*.dat"))


def test_flow_app_mixed_precision_rows(tmp_path):
    run = prepare(tmp_path, {"Precision": "fp32_12", "ReunitEvery": 5})
    subprocess.run([str(APP), str(run)], capture_output=True, text=True, check=True)
    got = (tmp_path / "out" / "flow" / "conf0001.dat").read_text().splitlines()
    exp = (GOLDEN / "app_flow" / "expected" / "flow" / "conf0001.dat").read_text().splitlines()
    assert len(got) == len(exp) and got[0] == exp[0]
    for a, b in zip(got[1:], exp[1:]):
        va, vb = [float(x) for x in a.split()], [float(x) for x in b.split()]
        assert va[0] == vb[0]
        assert abs(va[1] - vb[1]) < 2e-6 and abs(va[3] - vb[3]) < 1e-6 * abs(vb[3]) + 2e-6


def _pgfg(tmp_path, params, extra=None):
    import json

    cfg = {"App": {"type": "PGFG", "params": params},
           "LatticeSize": {"x": 4, "y": 4, "z": 4, "t": 4}, "SubLatticeSize": {"x": 4, "y": 4, "z": 4, "t": 4},
           "Action": {"type": "puregauge", "params": {"beta": 6.0}}, "Observables": ["superobs"],
           "OutputDir": str(tmp_path / "out")}
    cfg.update(extra or {})
    (tmp_path / "gen.json").write_text(json.dumps(cfg))
    return subprocess.run([str(APP), str(tmp_path / "gen.json")], capture_output=True, text=True, check=True)


@pytest.mark.parametrize("params,extra,therm_reports,saved_after", [
    # NConf 3 of 6 MC steps: a configuration every 2 sweeps, after 4 thermalisation sweeps
    ({"startType": "Cold", "MCSteps": 6, "thermSteps": 4, "SU3eps": 0.24, "NConf": 3}, {},
     [2, 4], [6, 8, 10]),
    # NCorr 4 of 6: NConf = 1, so 6 sweeps between configurations (the reference's integer arithmetic);
    # 3 thermalisation sweeps, no report; FP32 links, seed 5, big-endian files
    ({"startType": "Hot", "MCSteps": 6, "thermSteps": 3, "SU3eps": 0.3, "NCorr": 4},
     {"Precision": "fp32_18", "Seed": 5, "Endian": "big"}, [], [9]),
])
def test_generator_app_writes_the_seeded_chain(tmp_path, params, extra, therm_reports, saved_after):
    """The PGFG application: its thermalisation and sampling loops over the
    device Metropolis, each saved confNNNN.bin equal (bit for bit) to the same
    seeded chain run as one ymflow_generate_metropolis call, and its
    observables those of the saved field."""
    import numpy as np

    from latticeyangmills_b200 import GluonField, read_conf

    res = _pgfg(tmp_path, params, extra)
    out = tmp_path / "out"
    assert res.stdout.count("Thermalization Step") == len(therm_reports)
    for s in therm_reports:
        assert "Thermalization Step %4i\n" % s in res.stdout
    assert res.stdout.count("Configuration Number") == len(saved_after)
    assert res.stdout.count("\tAccept. Ratio = ") == len(therm_reports) + len(saved_after)
    rows = (out / "observables.dat").read_text().splitlines()
    assert rows[0] == "Step\tPlaq.\tTopc.\tEnerg.\t"
    k = saved_after[0] - params["thermSteps"]
    assert [r.split("\t")[0] for r in rows[1:]] == [str(k * (i + 1)) for i in range(len(saved_after))]
    full = np.loadtxt(out / "observables.full.dat", skiprows=1, ndmin=2)
    assert sorted(p.name for p in out.glob("conf*.bin")) == ["conf%04d.bin" % i for i in range(len(saved_after))]
    n = (4, 4, 4, 4)
    prec = extra.get("Precision", "fp64")
    big = extra.get("Endian") == "big"
    with GluonField(n, prec) as f:
        for i, total in enumerate(saved_after):
            acc = f.generate_metropolis(6.0, params["SU3eps"], total, 30, extra.get("Seed", 1),
                                        params["startType"].lower())
            want = f.download()
            got = read_conf(out / ("conf%04d.bin" % i), n, big_endian=big)
            assert np.array_equal(got, want), i
            o = f.observables()
            assert full[i, 2] == o.plaq and full[i, 3] == o.topc and full[i, 4] == o.energy
            assert abs(full[i, 5] - acc) <= 1e-14 * acc
            assert rows[i + 1].split("\t")[1] == "%f" % o.plaq
            assert "Configuration Number %4i\n\tPlaq.\t = %f \n" % (i, o.plaq) in res.stdout


def test_generated_configurations_flow_through_the_flow_app(tmp_path):
    """Generator then flow, both drop-in applications: the FLOW app reads the
    PGFG app's confNNNN.bin files and its first row is their plaquette."""
    import json

    import numpy as np

    _pgfg(tmp_path, {"startType": "Cold", "MCSteps": 4, "thermSteps": 2, "SU3eps": 0.24, "NConf": 2})
    full = np.loadtxt(tmp_path / "out" / "observables.full.dat", skiprows=1, ndmin=2)
    cfg = json.loads((GOLDEN / "app_flow" / "input.json").read_text()
                     .replace("@IN@", str(tmp_path / "out")).replace("@OUT@", str(tmp_path / "flowed")))
    (tmp_path / "flow.json").write_text(json.dumps(cfg))
    subprocess.run([str(APP), str(tmp_path / "flow.json")], capture_output=True, text=True, check=True)
    for i in range(2):
        rows = (tmp_path / "flowed" / "flow" / ("conf%04d.full.dat" % i)).read_text().splitlines()
        first = [float(x) for x in rows[1].split("\t")]
        assert first[2] == full[i, 2]
        last = [float(x) for x in rows[-1].split("\t")]
        assert last[2] > first[2]  # the flow smooths: the plaquette rises
