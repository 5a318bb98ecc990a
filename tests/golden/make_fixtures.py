"""Regenerate the golden fixtures in this folder from the reference checkout.

Run once in a container that holds the reference (read-only) checkout:

    python tests/golden/make_fixtures.py /path/to/reference

It writes
  * ``sample_msh.npz``  -- ``test_meshes/sample.msh`` (the reference's sweep
    benchmark mesh, 2,776 faces / 1,390 vertices) as vertices, 0-based faces
    and physical tags, read with the Gmsh 2.2 reader of
    ``beat_engine_b200.mesh`` (a restatement of ``load_gmsh22_with_tags``);
  * ``baseline_sweep_cpu.json`` -- the per-frequency ``pressure_norm`` /
    ``field_norm`` the reference's Julia CPU path produced for that mesh
    (``results/baseline_sweep_cpu.json``) plus the workload parameters of
    ``scripts/benchmark_sweep.jl:36-55``.

Nothing at test time reads the reference checkout; the tests read these files.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from beat_engine_b200.mesh import load_gmsh22_with_tags  # noqa: E402


def main(ref_root: str) -> None:
    jl = os.path.join(ref_root, "src", "beat_engine", "julia_local")
    mesh = load_gmsh22_with_tags(os.path.join(jl, "test_meshes", "sample.msh"), 1.0)
    np.savez_compressed(os.path.join(HERE, "sample_msh.npz"), vertices=mesh.vertices,
                        faces=mesh.faces, tags=mesh.physical_tags)
    with open(os.path.join(jl, "results", "baseline_sweep_cpu.json"), encoding="utf-8") as fh:
        base = json.load(fh)
    out = {
        "source": "src/beat_engine/julia_local/results/baseline_sweep_cpu.json",
        "workload": {
            "mesh": "test_meshes/sample.msh", "scale": 0.001, "precision": base["precision"],
            "quadrature_order": base["quadrature_order"], "singular_order": base["singular_order"],
            "sound_speed": 343.0, "rho": 1.21, "tag_throat": 2, "distance": 2.0,
            "eval_points": base["eval_points"], "symmetry": base["symmetry"],
            "julia_version": base["julia_version"], "git_commit": base["git_commit"],
        },
        "frequencies": [{k: row[k] for k in ("frequency_hz", "wavenumber", "pressure_norm", "field_norm")}
                        for row in base["frequencies"]],
        "ci_relative_tolerance": 1e-3,
    }
    with open(os.path.join(HERE, "baseline_sweep_cpu.json"), "w", encoding="utf-8") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
