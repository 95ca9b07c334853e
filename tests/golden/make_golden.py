"""Regenerate the golden fixtures of this directory from the reference tree.

Run in a container where the reference checkout exists (it is not needed to
run the tests):  python tests/golden/make_golden.py /path/to/jaxrens

Writes
  lj8_frames.json   the four frames of tests/_assets/data/lj8_npt/output/
                    lj8_npt.traj.extxyz (cell, positions, ns_energy = U_LJ +
                    0.1*V for LJ eps=sigma=1, rc=2.5, P=0.1) -- golden vectors
                    for the LJ backend + EnsembleTerm.
  lj8_energies.json header and first rows of lj8_npt.energies (format pin).
  prior_mass.json   outputs of the reference's numpy-only prior_mass.py
                    (log_alpha, iteration_offsets, log_dead_weights).
  thermo.json       outputs of the reference's numpy/scipy-only
                    postprocess/thermodynamics.py (log_evidence,
                    partition_function, heat_capacity) on seeded synthetic
                    dead/live energies.
"""

from __future__ import annotations

import importlib.util
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def frames(path):
    lines = open(path).read().splitlines()
    out, i = [], 0
    while i < len(lines):
        n = int(lines[i])
        hdr = lines[i + 1]
        lat = [float(v) for v in re.search(r'Lattice="([^"]+)"', hdr).group(1).split()]
        e = float(re.search(r"ns_energy=([-0-9.eE+]+)", hdr).group(1))
        it = int(re.search(r"iter=(\d+)", hdr).group(1))
        pos = [[float(v) for v in lines[i + 2 + k].split()[1:4]] for k in range(n)]
        out.append({"iter": it, "cell": lat, "positions": pos, "ns_energy": e})
        i += 2 + n
    return out


def main(ref_root: str) -> None:
    asset = os.path.join(ref_root, "tests/_assets/data/lj8_npt/output")
    fr = frames(os.path.join(asset, "lj8_npt.traj.extxyz"))
    meta = {"epsilon": 1.0, "sigma": 1.0, "cutoff": 2.5, "pressure": 0.1,
            "source": "tests/_assets/data/lj8_npt/output/lj8_npt.traj.extxyz"}
    json.dump({"meta": meta, "frames": fr}, open(os.path.join(HERE, "lj8_frames.json"), "w"), indent=1)
    en = open(os.path.join(asset, "lj8_npt.energies")).read().splitlines()
    json.dump({"header": en[0], "rows": en[1:21],
               "source": "tests/_assets/data/lj8_npt/output/lj8_npt.energies"},
              open(os.path.join(HERE, "lj8_energies.json"), "w"), indent=1)
    spec = importlib.util.spec_from_file_location(
        "ref_prior_mass", os.path.join(ref_root, "src/jaxrens/prior_mass.py"))
    pm = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(pm)
    cases = []
    for K, nc in [(128, 1), (512, 1), (1024, 1), (32, 1), (64, 4), (100, 7)]:
        xo, wo = pm.iteration_offsets(K, nc)
        cases.append({"n_live": K, "n_cull": nc, "log_alpha": pm.log_alpha(K, nc),
                      "x_offset": list(map(float, xo)), "w_offset": list(map(float, wo)),
                      "log_dead_weights_30": list(map(float, pm.log_dead_weights(30, K, nc))),
                      "log_live_weight_30": float(pm.log_live_weight(30, K, nc))})
    json.dump({"cases": cases, "source": "src/jaxrens/prior_mass.py"},
              open(os.path.join(HERE, "prior_mass.json"), "w"), indent=1)
    # thermodynamics.py imports only jaxrens.prior_mass: serve the module
    # loaded above under that name instead of importing the (JAX) package
    import types

    pkg = types.ModuleType("jaxrens")
    pkg.__path__ = []
    sys.modules.setdefault("jaxrens", pkg)
    sys.modules["jaxrens.prior_mass"] = pm
    spec = importlib.util.spec_from_file_location(
        "ref_thermo", os.path.join(ref_root, "src/jaxrens/postprocess/thermodynamics.py"))
    th = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(th)
    rng = np.random.default_rng(2024)
    tcases = []
    for K, nc, n_dead in [(32, 1, 300), (64, 3, 450)]:
        dead = np.sort(rng.normal(0.0, 3.0, n_dead))[::-1] + np.linspace(5.0, -5.0, n_dead)
        live = dead[-1] - np.abs(rng.normal(0.0, 0.5, K))
        betas = [0.2, 0.7, 1.0, 2.5]
        tcases.append({
            "n_live": K, "n_cull": nc, "dead": dead.tolist(), "live": live.tolist(),
            "betas": betas,
            "log_evidence": float(th.log_evidence(dead, live, K, nc)),
            "partition_function": [float(th.partition_function(b, dead, live, K, nc)) for b in betas],
            "heat_capacity": [float(th.heat_capacity(b, dead, live, K, nc)) for b in betas]})
    json.dump({"cases": tcases, "source": "src/jaxrens/postprocess/thermodynamics.py"},
              open(os.path.join(HERE, "thermo.json"), "w"), indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the jaxrens checkout>")
    main(sys.argv[1])
