"""Generates the golden fixtures of tests/golden/ by running the reference
itself (built from its sources by oracle/Makefile.ref into oracle/_ref/) on
synthetic models.

    make -f oracle/Makefile.ref
    python tests/golden/make_golden.py

Every fixture is one ``.npz`` holding the model parameters it was made from
and the reference's outputs: the integer maps of make_PartMesh_FW, the
assembled TMP_AIJ rows, the skyline profile and LDL^T factor of every
subdomain, the residual history, the converged edge solution and the
element results B, E, Je of the post step (also once with the first
Permittivity and Conductor flags left out).  The C1 fixture (hddm_eps
1e-10) keeps the residual history, the iteration count and the whole edge
solution; the C2 and C3 fixtures keep the initial norm and the residuals
of the first 10 and 3 interface iterations (hddm_max_loop 10 and 3).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from adventure_fullwave_b200 import meshgen  # noqa: E402
import refdump  # noqa: E402

# name -> (make_model kwargs, hddm_eps, hddm_max_loop, full dump)
CASES = {
    "tiny": (dict(name="tiny", n=4, size=1.0, npml=1, layers=None, nleaves=4, leaf_cap=None, jitter=None, seed=0),
             1e-12, 2000, True),
    "layered": (dict(name="layered", n=6, size=1.5, npml=1, layers=2, nleaves=None, leaf_cap=200,
                     jitter=(0.3, 0.7), seed=3), 1e-10, 4000, True),
    "c1": (dict(name="c1", seed=0), 1e-10, 40000, False),
    "c2_head": (dict(name="c2", seed=0), 1e-6, 10, False),
    "c3_head": (dict(name="c3", seed=0), 1e-6, 3, False),
    # element sources instead of the edge source: delta-gap voltages in a
    # conducting block, and an antenna current on a block of its own flag
    "gap": (dict(name="gap", n=4, size=1.0, npml=1, layers=None, nleaves=4, leaf_cap=None, jitter=None, seed=0),
            1e-12, 2000, True),
    "antenna": (dict(name="antenna", n=6, size=1.5, npml=1, layers=2, nleaves=None, leaf_cap=200,
                     jitter=(0.3, 0.7), seed=3), 1e-10, 4000, True),
}

EPS0 = 8.8541878128e-12


def add_element_source(model, kind: str) -> None:
    """The element source of the ``gap`` and ``antenna`` cases."""
    if kind == "gap":
        meshgen.add_region(model, (0.25, 0.25, 0.25), (0.75, 0.75, 0.75), EPS0, 50.0)
        # the second box holds one vertex of the first: the later gap wins there
        meshgen.delta_gap_source(model, [(0.24, 0.76, 0.24, 0.76, 0.49, 0.51), (0.49, 0.51, 0.49, 0.51, 0.49, 0.51)],
                                 [1.0, 2.0])
    elif kind == "antenna":
        f = meshgen.add_region(model, (0.5, 0.5, 0.5), (1.0, 1.0, 1.0), EPS0, 0.0)
        x, y, z = model.vertex_crd.T
        jo = np.stack([0.1 * x, -0.2 * y, 1.0 + 0.5 * z], axis=1)
        jor = np.stack([np.full_like(x, 0.05), 0.3 * x, np.full_like(x, -0.7)], axis=1)
        meshgen.antenna_source(model, [f], jo[None], jor[None])
    else:
        raise ValueError(kind)
    model.sources = []


def build_model(params: dict):
    """The model a fixture was made from (its parameters as stored)."""
    model = meshgen.make_model(**params["kw"])
    if params.get("element_source"):
        add_element_source(model, params["element_source"])
    meshgen.round_trip_material(model)
    return model


def make_case(name: str) -> str:
    kw, eps, maxloop, full = CASES[name]
    params = dict(kw=kw, eps=eps, max_loop=maxloop)
    if name in ("gap", "antenna"):
        params["element_source"] = name
    model = build_model(params)
    out = refdump.run_harness(model, eps, maxloop, dump=2 if full else 0)
    arrays = {
        "params": np.frombuffer(json.dumps(params).encode(), dtype=np.uint8),
        "hist": out["hist"],
        "norm0": np.array([out["norm0"]]),
        "hist_full": out["hist_full"],
        "norm0_full": np.array([out["norm0_full"]]),
        "iterations": np.array([out["json"]["iterations"]]),
        "total_free": np.array([out["json"]["total_free"]]),
    }
    if full:
        arrays["x"] = out["x"]
        for tag in ("post", "post_drop"):
            for k, v in zip(("B", "E", "Je"), out[tag]):
                arrays[f"{tag}_{k}"] = v
        for s, (im, am, fm) in enumerate(zip(out["ints"], out["aij"], out["fac"])):
            for k, v in im.items():
                arrays[f"s{s}_{k}"] = v
            for k, v in am.items():
                arrays[f"s{s}_aij_{k}"] = v
            arrays[f"s{s}_idx1"] = fm["idx1"]
            arrays[f"s{s}_idx2"] = fm["idx2"]
            arrays[f"s{s}_fac"] = fm["mat"]
    elif name == "c1":
        arrays["x"] = out["x"]
    path = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(path, **arrays)
    return path


def params_of(npz) -> dict:
    return json.loads(bytes(npz["params"]).decode())


if __name__ == "__main__":
    for name in (sys.argv[1:] or CASES):
        print(make_case(name), os.path.getsize(os.path.join(HERE, f"ref_{name}.npz")))
