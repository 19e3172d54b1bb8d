"""Generate tests/golden/golden.json from the COMPILED REFERENCE (oracle/_ref).

Each case builds a seeded synthetic state (aturan_b200.state.synthetic_state, deterministic
numpy), loads it into the reference model, runs the reference's own routine(s) and records, per
output field, the SHA-256 of the FP64 bytes plus a seeded sample of cell values (hex). The
oracle restatement must reproduce every digest bit for bit (tests/test_golden.py), which pins
it on machines without the reference tree.

    python tests/golden/make_golden.py          # needs oracle/_ref (make -C oracle ref)
    python tests/golden/make_golden.py post_step   # (re)make the named cases, keep the others
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from aturan_b200 import fields as F, params as P, state as S  # noqa: E402

CASES = {
    "satadj4": dict(seed=101, outputs=["t"] + [n for g in F.GASES for n in F.GAS_FIELDS[g]]),
    "rk4": dict(seed=102, outputs=F.PROGNOSTIC + ["p_hydro", "p_bfollow"] + F.PROJECTION + ["buoy_ref_level"]),
    "pressure_gs": dict(seed=103, outputs=["p_dyn", "aux_u", "aux_v", "aux_w"]),
    "pressure_rb3": dict(seed=104, outputs=["p_dyn"] + F.PROJECTION),
    "step_gs": dict(seed=105, outputs=F.PROGNOSTIC + ["p_dyn", "p_hydro", "p_bfollow"] + F.PROJECTION),
    # the moist convective adjustment with the default knobs
    "mca": dict(seed=107, outputs=["t", "nh4sh"] + [n for g in F.GASES for n in F.GAS_FIELDS[g]]),
    # the passes after RK4 with the default knobs, on post_case.post_state(state, seed + 1)
    "post_step": dict(seed=106, outputs=["t", "u", "v", "w", "h2o", "h2o_cloud", "h2o_ice", "h2s", "h2s_cloud",
                                         "h2s_ice", "nh3", "nh3_cloud", "nh3_ice", "ch4", "ch4_cloud", "ch4_ice",
                                         "nh4sh", "massflux_h2s", "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh",
                                         "thermalmassflux"]),
    # the chemistry (equilibrium form, default knobs) on chem_case.chem_state(state, seed + 1)
    "chem_eq": dict(seed=108, outputs=["t", "nh3", "h2s", "nh4sh"]),
    "chem_forcing": dict(seed=109, outputs=["rho_mix", "difflux_h2s", "difflux_nh3", "difflux_nh4sh", "massflux_h2s",
                                            "massflux_nh3", "massflux_nh4sh", "fluxlim_nh4sh", "thermalmassflux"]),
    # the turbulence closure (k-omega SST, default knobs) on turb_case.turb_state(state, seed + 1)
    "turbulence": dict(seed=110, outputs=["tke", "dis", "nue", "prod", "tke_source", "dis_source", "tken", "disn"]),
    # the precipitation (default knobs) on precip_case.precip_state(state, seed + 1)
    "precipitation": dict(seed=111, outputs=["Q_precip", "S_precip_ch4", "S_precip_ch4_cloud", "S_precip_ch4_ice",
                                             "S_precip_h2o", "S_precip_h2o_cloud", "S_precip_h2o_ice",
                                             "S_precip_h2s", "S_precip_h2s_cloud", "S_precip_h2s_ice",
                                             "S_precip_nh3", "S_precip_nh3_cloud", "S_precip_nh3_ice"]),
}
NSAMPLE = 32


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def samples(a, seed):
    rng = np.random.default_rng(seed)
    flat = np.ascontiguousarray(a, dtype=np.float64).ravel()
    idx = rng.integers(0, flat.size, NSAMPLE)
    return [[int(i), float.hex(float(flat[i]))] for i in idx]


def run_case(name, runner):
    """runner(state) -> dict of outputs; returns the golden record."""
    c = CASES[name]
    p = P.default_params()
    st = S.synthetic_state(p, seed=c["seed"])
    out = runner(name, p, st)
    rec = {"seed": c["seed"], "fields": {}}
    for n in c["outputs"]:
        rec["fields"][n] = {"sha256": digest(out[n]), "samples": samples(out[n], c["seed"] + len(n))}
    return rec


def post_input(p, st, seed):
    from tests.post_case import post_state
    return post_state(st, p, seed + 1)


def chem_input(p, st, seed):
    from tests.chem_case import chem_state
    return chem_state(st, p, seed + 1)


def turb_input(p, st, seed):
    from tests.turb_case import turb_state
    return turb_state(st, p, seed + 1)


def precip_input(p, st, seed):
    from tests.precip_case import precip_state
    return precip_state(st, p, seed + 1)


def ref_runner(name, p, st):
    from oracle.ref import Ref
    ref = Ref.get_instance()
    if name == "post_step":
        st = post_input(p, st, CASES[name]["seed"])
    if name.startswith("chem_"):
        st = chem_input(p, st, CASES[name]["seed"])
    if name == "turbulence":
        st = turb_input(p, st, CASES[name]["seed"])
    if name == "precipitation":
        st = precip_input(p, st, CASES[name]["seed"])
    ref.load(st)
    if name == "satadj4":
        for g in range(4):
            ref.satadj(g)
    elif name == "rk4":
        ref.rk4()
    elif name == "pressure_gs":
        ref.pressure_gs()
    elif name == "pressure_rb3":
        ref.pressure_rb(3)
    elif name == "step_gs":
        ref.pressure_gs()
        for g in range(4):
            ref.satadj(g)
        ref.sync_ncopies()
        ref.rk4()
    elif name == "post_step":
        ref.post_step(P.default_post_params())
    elif name == "mca":
        ref.mca()
    elif name == "chem_eq":
        ref.chem_eq()
    elif name == "chem_forcing":
        ref.chem_forcing()
    elif name == "turbulence":
        ref.turbulence()
    elif name == "precipitation":
        ref.precipitation()
    out = ref.state([n for n in CASES[name]["outputs"] if n != "buoy_ref_level"])
    if "buoy_ref_level" in CASES[name]["outputs"]:
        out["buoy_ref_level"] = ref.get("buoy_ref_level")
    return out


def main(only=()):
    path = os.path.join(HERE, "golden.json")
    golden = {"note": "SHA-256 of FP64 outputs of the compiled reference on seeded synthetic states; "
                      "made by tests/golden/make_golden.py",
              "numpy": np.__version__, "cases": {}}
    if only and os.path.exists(path):
        golden["cases"] = json.load(open(path))["cases"]
    for name in (only or CASES):
        golden["cases"][name] = run_case(name, ref_runner)
        print("done", name, flush=True)
    with open(path, "w") as fh:
        json.dump(golden, fh, indent=1)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
