"""Replay of the recorded vortex-diagnostics calls (tests/golden/diagnostics.npz)
against an implementation: the oracle on the CPU or the device module."""
import json
import math

import numpy as np

from oracle import lh82 as O


def diag_states(golden_dir):
    """name -> (u, v, z, dx, recorded calls) for the three fixture states."""
    g = np.load(golden_dir / "diagnostics.npz")
    ps = np.load(golden_dir / "production_storm.npz")
    vt = np.load(golden_dir / "vortex_tracker.npz")
    res = json.loads(str(g["results_json"]))
    fields = {"storm": (ps["s4_u"], ps["s4_v"]), "tracker": (vt["exp_u"], vt["exp_v"]),
              "deep": (g["c_u"], g["c_v"])}
    out = {}
    for name, r in res.items():
        z = O.build_base_state(r["nz"], r["Lz"])[0]
        out[name] = (*fields[name], z, r["dx"], r["calls"])
    return out


def replay(call, mod, u, v, z, dx):
    """Run one recorded call through ``mod`` (functions taking u, v, z in the
    oracle's keyword form)."""
    fn, kw = call["fn"], dict(call["kw"])
    zz = None if kw.pop("no_base", False) else z
    if fn == "compute_diagnostics":
        th = kw.pop("theta_xy_m")
        d = mod.compute_diagnostics(u, v, z, kw["cx_m"], kw["cy_m"], dx, dx, kw["u_env"],
                                    kw["v_env"], theta_xy_m=tuple(th), r_vent_m=kw["r_vent_m"])
        return d
    if fn == "format_diag_line":
        th = kw.pop("theta_xy_m")
        d = mod.compute_diagnostics(u, v, z, kw["cx_m"], kw["cy_m"], dx, dx, kw["u_env"],
                                    kw["v_env"], theta_xy_m=tuple(th), r_vent_m=kw["r_vent_m"])
        return mod.format_diag_line(d)
    if fn == "vorticity_center":
        return mod.vorticity_center(u, v, kw["cx_m"], kw["cy_m"], dx, dx, z=zz,
                                    window_m=kw["window_m"], z_top_m=kw["z_top_m"])
    if fn == "low_level_vmax":
        return mod.low_level_vmax(u, v, z, kw["cx_m"], kw["cy_m"], dx, dx, kw["u_env"],
                                  kw["v_env"], z_top_m=kw["z_top_m"])
    if fn == "vmax_3d":
        return mod.vmax_3d(u, v, z, kw["u_env"], kw["v_env"])
    if fn == "ventilation_flow":
        extra = {k: kw[k] for k in ("z_lo_m", "z_hi_m") if k in kw}
        return mod.ventilation_flow(u, v, kw["cx_m"], kw["cy_m"], dx, dx, z=zz,
                                    r_vent_m=kw["r_vent_m"], n_bins=kw["n_bins"],
                                    u_env=kw.get("u_env"), v_env=kw.get("v_env"), **extra)
    if fn == "perturbation_ke":
        return mod.perturbation_ke(u, v, kw["u_env"], kw["v_env"])
    if fn == "enstrophy":
        return mod.enstrophy(u, v, dx, dx, z=z, z_top_m=kw["z_top_m"])
    if fn == "subcell_refine":
        return list(mod.subcell_refine(u, v, kw["x_m"], kw["y_m"], dx, patch=kw["patch"]))
    raise KeyError(fn)


def same(a, b, rtol=0.0):
    """Equal, NaN equal to NaN; floats within rtol relative (0: exact)."""
    if isinstance(b, dict):
        return isinstance(a, dict) and set(a) == set(b) and all(
            same(a[k], b[k], rtol) for k in b)
    if isinstance(b, (list, tuple)):
        return len(a) == len(b) and all(same(x, y, rtol) for x, y in zip(a, b))
    if isinstance(b, str):
        return a == b
    a, b = float(a), float(b)
    if math.isnan(b):
        return math.isnan(a)
    return a == b or abs(a - b) <= rtol * max(abs(b), 1e-300)
