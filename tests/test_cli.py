"""The command line (cli.py): P1 CIF and kUPS-style YAML inputs (the reference's formats,
src/structure.jl:37-92, src/forcefield.jl:54-101) into a FrameworkBatch, replication to the
cutoff guard, argument errors; on a B200 its JSON results equal a widom call on the same inputs."""
import io
import json
import os
import subprocess
import sys

import numpy as np
import pytest

CIF = """data_test
_symmetry_space_group_name_H-M 'P 1'
_cell_length_a 13.0
_cell_length_b 13.5
_cell_length_c 14.0
_cell_angle_alpha 90
_cell_angle_beta 90
_cell_angle_gamma 90
loop_
_atom_site_label
_atom_site_type_symbol
_atom_site_fract_x
_atom_site_fract_y
_atom_site_fract_z
_atom_site_charge
Zn1 Zn 0.10 0.20 0.30 0.60
O1 O 0.55 0.25 0.35 -0.30
O2 O 0.30 0.70 0.60 -0.30
C1 C 0.80 0.80 0.10 0.00
"""

FF = """cutoff: 6.0
tail_correction: false
parameters:
  Zn_: [2.46, 0.0054]
  O_: [3.12, 0.0052]
  C_: [3.43, 0.0045]
  C_co2: [2.80, 0.0023]
  O_co2: [3.05, 0.0068]
"""

GUEST = """positions: [[0.0, 0.0, 0.0], [1.16, 0.0, 0.0], [-1.16, 0.0, 0.0]]
symbols: [C_co2, O_co2, O_co2]
charges: [0.70, -0.35, -0.35]
critical_temperature: 304.13
critical_pressure: 7_377_300
acentric_factor: 0.224
"""


@pytest.fixture
def files(tmp_path):
    paths = {}
    for name, text in (("fw.cif", CIF), ("ff.yaml", FF), ("co2.yaml", GUEST)):
        p = tmp_path / name
        p.write_text(text)
        paths[name] = str(p)
    return paths


def args_for(files, *extra):
    return ["widom", "--cif", files["fw.cif"], "--forcefield", files["ff.yaml"], "--guest", files["co2.yaml"],
            "--T", "298.15", "--ninsert", "20000", *extra]


def test_inputs_and_replication(pa, files):
    a = pa.cli.parser().parse_args(args_for(files))
    fws, ff, guest, ewald = pa.cli.build_inputs(a)
    # 2 (6 + 1.16) = 14.32 A between opposite faces: every axis doubles
    assert fws[0].replication == (2, 2, 2) and len(fws[0].frac) == 32
    assert ewald.cutoff == 6.0 and not ff.tail
    assert list(guest.types) == [ff.typeindex("C_co2"), ff.typeindex("O_co2"), ff.typeindex("O_co2")]
    assert guest.pc == 7377300.0
    a = pa.cli.parser().parse_args(args_for(files, "--replicate", "3", "2", "2", "--ewald-cutoff", "6.5", "--float32"))
    fws, ff, guest, ewald = pa.cli.build_inputs(a)
    assert fws[0].replication == (3, 2, 2) and fws[0].T == np.float32 and ewald.cutoff == 6.5
    batch = pa.FrameworkBatch(fws, ff, guest, ewald, T=np.float32)
    assert batch.nsys == 1 and len(batch.positions) == 48


def test_argument_errors(pa, files, capsys):
    with pytest.raises(SystemExit):
        pa.cli.parser().parse_args(["widom", "--cif", files["fw.cif"]])
    # a replication below the guard is the batch's own error, reported as one line
    rc = pa.cli.main(args_for(files, "--replicate", "1", "1", "1"))
    assert rc == 2 and "replicate it by" in capsys.readouterr().err


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [(), ("--float32",)])
def test_results_equal_widom(pa, backend, files, extra):
    out = io.StringIO()
    assert pa.cli.main(args_for(files, "--seed", "5", *extra), out=out) == 0
    rec = json.loads(out.getvalue().strip().splitlines()[0])
    a = pa.cli.parser().parse_args(args_for(files, *extra))
    fws, ff, guest, ewald = pa.cli.build_inputs(a)
    T = np.float32 if extra else np.float64
    r = pa.widom(pa.FrameworkBatch(fws, ff, guest, ewald, T=T), guest, T=298.15, ninsert=20000, seed=5,
                 backend=backend)[0]
    assert rec["K_H"] == r.K_H and rec["mu_ex_eV"] == r.mu_ex and rec["q_st_eV"] == r.q_st


@pytest.mark.gpu
def test_module_entry(files):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, os.path.join(root, "pureadsorb.jl_b200"), *args_for(files)],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    rec = json.loads(p.stdout.strip().splitlines()[0])
    assert rec["nsamples"] == 20000 and rec["K_H"] > 0


def test_two_frameworks_each_replicated(pa, files, tmp_path):
    # a second, larger CIF: each framework gets its own smallest replication that passes the guard
    big = CIF.replace("_cell_length_a 13.0", "_cell_length_a 29.0")
    p = tmp_path / "big.cif"
    p.write_text(big)
    a = pa.cli.parser().parse_args(args_for(files) + ["--cif", str(p)])
    fws, ff, guest, ewald = pa.cli.build_inputs(a)
    assert [fw.replication for fw in fws] == [(2, 2, 2), (1, 2, 2)]
    batch = pa.FrameworkBatch(fws, ff, guest, ewald)
    assert batch.nsys == 2 and batch.nframeworks() == 2
