"""Shared helpers: golden case loading and conversion to oracle specs."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import ref_numpy as rn  # noqa: E402


def load_cases():
    with open(GOLDEN / "cases.json") as fh:
        return json.load(fh)


def box_mask(shape, box):
    m = np.zeros(shape, dtype=bool)
    (a0, a1), (b0, b1), (c0, c1) = box
    m[a0:a1, b0:b1, c0:c1] = True
    return m


def eps_from_case3d(case):
    shape = tuple(case["size"])
    return rn.build_eps_r(shape, [(box_mask(shape, m["box"]), m["epsilon_r"])
                                  for m in case["materials"]])


def oracle3d_from_case(case, dtype=np.float64):
    shape = tuple(case["size"])
    srcs = [dict(position=tuple(s["position"]), polarization=s["polarization"],
                 amplitude=s["amplitude"], kind="sine", frequency=s["frequency"])
            for s in case["sources"]]
    spec = rn.Spec3D(size=shape, dx=case["resolution"], boundary=case["boundary"],
                     pml_layers=case["pml_layers"], eps_r=eps_from_case3d(case), sources=srcs)
    dt = rn.default_dt_3d(case["resolution"])
    n = rn.n_steps_from_span(case["t_span"], dt)
    o = rn.Oracle3D(spec, dt=dt, t_start=case["t_span"][0], dtype=dtype)
    return o, n


def oracle2d_from_case(case, dtype=np.float64):
    srcs = [dict(y=s["y"], amplitude=s["amplitude"], kind="sine", frequency=s["frequency"])
            for s in case["sources"]]
    walls = [(w["y"], w["gap_start"], w["gap_end"]) for w in case["walls"]]
    spec = rn.Spec2D(size=tuple(case["size"]), dx=case["resolution"], boundary=case["boundary"],
                     pml_layers=case["pml_layers"], sources=srcs, walls=walls)
    dt = rn.default_dt_2d(case["resolution"])
    n = rn.n_steps_from_span(case["t_span"], dt)
    return rn.Oracle2D(spec, dt=dt, t_start=case["t_span"][0], dtype=dtype), n


def golden(kind, name):
    return dict(np.load(GOLDEN / f"ref{kind}_{name}.npz"))
