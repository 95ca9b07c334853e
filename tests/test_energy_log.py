"""The .energies writer (CPU): the reference's format, pinned by the lj8
fixture, bulk rows from info buffers."""

import json
import os

import numpy as np

from jaxrens_b200.energy_log import EnergyLogger, dead_point_rows

GOLD = os.path.join(os.path.dirname(__file__), "golden", "lj8_energies.json")


def test_writer_reproduces_the_reference_fixture_rows(tmp_path):
    g = json.load(open(GOLD))
    n_walkers, n_cull, n_dof, _, n_atoms = g["header"].split()
    rows = [r.split() for r in g["rows"]]
    path = tmp_path / "run.energies"
    lg = EnergyLogger(path, int(n_walkers), int(n_cull), int(n_dof), int(n_atoms))
    for it, e, v in rows:
        lg.write_entry(int(it), float(np.float32(float(e))), float(np.float32(float(v))))
    lg.close()
    text = open(path).read().splitlines()
    assert text[0] == g["header"]
    assert text[1:] == g["rows"]
    log = EnergyLogger.read(path)
    assert (log.n_walkers, log.n_cull, log.n_atoms) == (32, 1, 8)
    assert len(log.iterations) == len(rows)


def test_bulk_rows_one_per_cull_in_descending_order(tmp_path):
    e = np.array([[5.0, 4.0, 3.5], [3.0, 2.5, 2.0]])           # (n_iter, n_cull)
    c = np.zeros((2, 3, 3, 3), np.float32)
    for q in range(3):
        c[:, :, q, q] = 2.0
    its, ens, vols = dead_point_rows(7, e, c)
    assert its.tolist() == [7, 7, 7, 8, 8, 8]
    assert ens.tolist() == e.reshape(-1).tolist()
    assert np.allclose(vols, 8.0)
    lg = EnergyLogger(tmp_path / "m.energies", 16, 3, 0, 4)
    lg.write_entries(its, ens, vols)
    lg.close()
    lines = open(tmp_path / "m.energies").read().splitlines()
    assert lines[0] == "16 3 0 0.0 4" and lines[1] == "7 5.0000000000e+00 8.0000000000e+00"
