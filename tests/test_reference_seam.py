"""The reference-side seam, applied to the reference package itself.

INTEGRATION.md gives the block a maintainer adds at the top of
``oracle_v8/__init__.py`` to switch a run to this backend.  This test takes
that block verbatim from INTEGRATION.md, applies it to a copy of the
reference's ``oracle_v8`` package (its Python files only; the reference tree
itself is read, never written), and imports the reference's own modules in a
fresh interpreter with ``ORACLE_BACKEND=b200``:

* ``from oracle_v8.solver import RK3Integrator, OperatorConfig, ...`` returns
  the B200 classes;
* the reference's ``production_config.build_production_config``
  (production_config.py:128-150) builds its OperatorConfig from B200
  components, and the B200 engine compiles it into a device plan spec with
  every production slot set;
* the run loops' modules (run_storm.py:32-49) import, and their read-outs
  (``oracle_v8.diagnostics``, ``oracle_v8.storm_tracker``) are the B200 ones.

No GPU is needed: nothing here creates a plan.  The reference tree is found
through ``ORACLE_V8_REF`` or as a ``reference`` directory beside this
repository; without it the test is skipped.
"""
import json
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _reference_root():
    cands = [os.environ.get("ORACLE_V8_REF"), str(ROOT.parent / "reference")]
    for c in cands:
        if c and (Path(c) / "oracle_v8" / "__init__.py").exists():
            return Path(c)
    return None


def _shim_block():
    md = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r"```python\n(# oracle_v8/__init__\.py.*?)```", md, re.S)
    assert m, "INTEGRATION.md has no oracle_v8/__init__.py shim block"
    return m.group(1)


_PROBE = r"""
import json, sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(1, sys.argv[2])
out = {}
from oracle_v8.solver import (RK3Integrator, OperatorConfig, AdvectionComponent,
                              AnelasticProjection, StepDiagnostics, State)
out["solver"] = [c.__module__ for c in (RK3Integrator, OperatorConfig, AdvectionComponent,
                                        AnelasticProjection, StepDiagnostics, State)]
from oracle_v8.grid.staggering import LorenzStaggering
out["grid"] = LorenzStaggering.__module__
from oracle_v8 import production_config as PC
out["production_config_file"] = PC.__file__
cfg = PC.build_production_config(64, 48, 16, 640e3, 480e3, 16e3, 5e-5, -3.0, 1.0)
out["config"] = {k: type(getattr(cfg, k)).__module__ for k in
                 ("projection", "advection", "coriolis", "surface_drag", "horiz_diffusion",
                  "divergence_damping", "newtonian_cooling")}
from oraclev8_b200.production_config import BaseState
from oraclev8_b200.solver.integrator import compile_config
spec = compile_config(cfg, BaseState(16, 16e3), "fp64")
out["spec"] = dict(projection=bool(spec.projection), advection=int(spec.advection),
                   coriolis=int(spec.coriolis), drag=bool(spec.drag),
                   diffusion=int(spec.diffusion), damping=bool(spec.damping),
                   cooling=bool(spec.cooling), u_env=float(spec.u_env), nx=spec.nx, ny=spec.ny)
from oracle_v8 import diagnostics as dg, storm_tracker as trk
from oracle_v8.backend import xp, wrap_base, to_numpy
out["readouts"] = [dg.vorticity_center.__module__, trk.find_storm_centre.__module__,
                   wrap_base.__module__]
import oracle_v8.run_storm as rs
out["run_storm"] = [rs.RK3Integrator.__module__, rs.IntensityCapComponent.__module__]
print(json.dumps(out))
"""


def test_shim_switches_the_reference_package_to_this_backend(tmp_path):
    ref = _reference_root()
    if ref is None:
        pytest.skip("reference tree not available (set ORACLE_V8_REF)")
    pkg = tmp_path / "oracle_v8"
    shutil.copytree(ref / "oracle_v8", pkg,
                    ignore=lambda d, names: [n for n in names if not (
                        n.endswith(".py") or (Path(d) / n).is_dir()) or n in (
                        "Logs", "__pycache__")])
    init = pkg / "__init__.py"
    init.write_text(_shim_block() + init.read_text())
    env = dict(os.environ, ORACLE_BACKEND="b200", ORACLE_GPU="0", PYTHONDONTWRITEBYTECODE="1")
    r = subprocess.run([sys.executable, "-c", _PROBE, str(tmp_path), str(ROOT)],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(m.startswith("oraclev8_b200.solver") for m in out["solver"]), out["solver"]
    assert out["grid"] == "oraclev8_b200.grid.staggering"
    # the reference's own config builder, now building B200 components
    assert out["production_config_file"].startswith(str(tmp_path))
    assert all(m.startswith("oraclev8_b200.") for m in out["config"].values()), out["config"]
    sp = out["spec"]
    assert sp["projection"] and sp["drag"] and sp["damping"] and sp["cooling"]
    assert sp["advection"] == 1 and sp["coriolis"] == 2 and sp["diffusion"] == 2
    assert sp["u_env"] == -3.0 and (sp["nx"], sp["ny"]) == (64, 48)
    assert out["readouts"] == ["oraclev8_b200.diagnostics", "oraclev8_b200.storm_tracker",
                               "oraclev8_b200.backend"]
    assert all(m.startswith("oraclev8_b200.") for m in out["run_storm"]), out["run_storm"]
