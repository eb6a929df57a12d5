"""The `fip` command line (fip_b200/fip, the reference's headless main() on the C ABI) against the
reference binary on the same parameter file: the stdout sampling CSV, the save_state dump files
(names and contents) and the stderr timing line `Finished N iterations after S s (x s/it)`
(src/main.cpp:204-263). Also: `quiet` handles print no loader warnings.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import refbin
from golden_util import Golden

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIP = os.path.join(ROOT, "fip_b200", "fip")


def _dump_names(prefix):
    """Dump files under `prefix` without their wall-clock stamp: (kind, int time)."""
    base = os.path.basename(prefix)
    out = set()
    for f in glob.glob(prefix + "_*"):
        rest = os.path.basename(f)[len(base) + 1:]
        for kind in refbin.KINDS:
            if rest.startswith(kind + "_"):
                t = rest[len(kind) + 1:].split("_")[0]
                if t.isdigit():
                    out.add((kind, int(t)))
    return out


@pytest.mark.parametrize("case", ["g1_wet_q_open", "g0_z_open_close"])
def test_cli_matches_reference_binary(case, tmp_path):
    if refbin.binary("fip_ref_nomask") is None:
        pytest.skip("oracle/_ref/fip_ref_nomask not built (make -f oracle/ref.mk REF=<reference sources>)")
    assert os.access(FIP, os.X_OK), "fip_b200/fip not built (make -C fip_b200/csrc)"
    g = Golden(case)
    y_ref = g.materialize(str(tmp_path / "ref"))
    y_fip = g.materialize(str(tmp_path / "fip"))
    ref = refbin.run("fip_ref_nomask", y_ref)
    p = subprocess.run([FIP, y_fip], cwd=str(tmp_path / "fip"), capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    # stderr: the same timing line, the same iteration count
    fin = refbin.parse_finished(p.stderr)
    assert fin is not None, p.stderr
    assert fin[0] == ref["iterations"]
    assert p.stderr.strip().splitlines()[-1].startswith(f"Finished {fin[0]} iterations after ")
    # stdout: the sampling CSV, same header text, same rows within the gates
    ra = [r for r in ref["stdout"].split("\n") if r]
    rb = [r for r in p.stdout.split("\n") if r]
    assert len(ra) == len(rb)
    if ra:
        assert ra[0] == rb[0]
        for a, b in zip(ra[1:], rb[1:]):
            va = [float(x) for x in a.split(";") if x]
            vb = [float(x) for x in b.split(";") if x]
            assert va[0] == vb[0] and np.allclose(va[1:], vb[1:], atol=1e-4, rtol=1e-6), (a, b)
    # dumps: the same files (up to the wall-clock stamp), contents within the gates
    name = os.path.basename(g.meta["name"])
    pa, pb = str(tmp_path / "ref" / name), str(tmp_path / "fip" / name)
    assert _dump_names(pa) == _dump_names(pb) and _dump_names(pa)
    da, db = refbin.dumps(pa), refbin.dumps(pb)
    for key in da:
        d = np.abs(da[key].astype(np.float64) - db[key].astype(np.float64))
        assert np.all(d <= 1e-4 + 1e-6 * np.abs(da[key])), (key, float(d.max()))


def test_quiet_handle_prints_no_loader_warnings(tmp_path, capfd):
    from fip_b200 import Simulation, synth

    sc = synth.scenario0(str(tmp_path), W=64, H=48, duration=2.0, save_every=0, name="q")
    with Simulation(sc.yaml_path, quiet=True) as sim:
        sim.step(2)
    assert "Warning" not in capfd.readouterr().err
    with Simulation(sc.yaml_path, quiet=False) as sim:
        sim.step(1)
    assert "Warning: no save_state times given" in capfd.readouterr().err
