"""The Python drop-in glue, run against the reference itself.

The integration recipe shadows eight ``magic_torch.sht`` functions and
``get_nl`` with this package's (the reference's own SHTns shadowing slot,
magic_torch/step_time.py:28-41) and calls ``configure_from_reference()`` in a
process that has imported ``magic_torch``.  These tests do exactly that in a
subprocess (the reference fixes its configuration at import, so one process
per configuration) on the reference's CPU path, and check:

* every name the recipe imports exists in both modules, and this package's
  positional parameters start with the reference's (same names, same order;
  extra trailing keywords are allowed);
* ``configure_from_reference()`` copies every size, factor and radial profile
  that the reference's get_nl, get_nl_anel and courant_check read at import
  (magic_torch/get_nl.py:12-17, get_nl_anel.py:12-20, courant.py:9-14),
  bit for bit, on a Boussinesq and on an anelastic configuration.

They need the reference's source tree (``MAGIC_TORCH_SRC``, default the
checkout this build reads) and skip where it is absent; no kernel runs.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = os.environ.get("MAGIC_TORCH_SRC", "/root/reference/src")

pytestmark = pytest.mark.skipif(
    not os.path.isfile(os.path.join(REF_SRC, "magic_torch", "config.py")),
    reason="reference source tree not present")

RECIPE_SHT = ("scal_to_spat", "scal_to_SH", "torpol_to_spat", "spat_to_sphertor",
              "torpol_to_curl_spat", "pol_to_grad_spat", "pol_to_curlr_spat",
              "torpol_to_dphspat")
OTHER_SHT = ("spat_to_SH", "scal_to_grad_spat", "sphtor_to_spat", "spat_to_qst")

WORKER = r"""
import inspect, json, sys
ref, root, cfg = sys.argv[1], sys.argv[2], json.loads(sys.argv[3])
sys.path[:0] = [ref, root]
from magic_torch.config import configure
configure(cfg)
import magic_torch.params as P
import magic_torch.pre_calculations as pc
import magic_torch.radial_functions as rf
import magic_torch.radial_scheme as rs
import magic_torch.sht as rsht
import magic_torch.get_nl as rnl
import magic_torch.get_nl_anel as rnla
import magic_torch.courant as rcour
import magic_b200
import magic_b200.sht as bsht
import magic_b200.get_nl as bnl
from magic_b200 import config as bc

def params(f):
    return [p.name for p in inspect.signature(f).parameters.values()
            if p.default is inspect.Parameter.empty]

def allparams(f):
    return [p.name for p in inspect.signature(f).parameters.values()]

magic_b200.configure_from_reference()
out = {"sig": {}, "cfg": {}, "prof": {}}
pairs = [(getattr(rsht, n, None), getattr(bsht, n, None), n) for n in json.loads(sys.argv[4])]
pairs += [(rnl.get_nl, bnl.get_nl, "get_nl"), (rnla.get_nl_anel, bnl.get_nl_anel, "get_nl_anel"),
          (rcour.courant_check, bnl.courant_check, "courant_check")]
for rf_, bf_, n in pairs:
    if rf_ is None or bf_ is None:
        out["sig"][n] = ["missing", rf_ is None, bf_ is None]
        continue
    out["sig"][n] = [params(rf_), allparams(bf_)]
out["cfg"] = dict(l_max=[P.l_max, bc.get("l_max")], minc=[P.minc, bc.get("minc")],
                  LFfac=[float(pc.LFfac), bc.lffac()], opm=[float(pc.opm), bc.get("opm")],
                  ViscHeatFac=[float(rf.ViscHeatFac), bc.get("ViscHeatFac")],
                  OhmLossFac=[float(rf.OhmLossFac), bc.get("OhmLossFac")])
n_r = P.n_r_max
for k, src in [("r", rs.r)] + [(k, getattr(rf, k)) for k in
        ("or1", "or2", "or4", "orho1", "orho2", "beta", "otemp1", "visc", "lambda_",
         "delxr2", "delxh2")]:
    got = bc.profile(k, n_r)
    out["prof"][k] = bool(got.shape == src.shape and (got == src.to(got.dtype)).all())
print("RESULT " + json.dumps(out))
"""

CONFIGS = {
    "bouss": {"l_max": 16, "minc": 1, "n_r_max": 9, "ek": 1e-3, "ra": 1e5, "pr": 1.0,
              "prmag": 5.0, "mode": 0},
    "anel": {"l_max": 8, "minc": 1, "n_r_max": 9, "strat": 5.0, "polind": 2.0, "g0": 0.0,
             "g1": 0.0, "g2": 1.0, "mode": 0, "ek": 1e-4, "ra": 3e6, "prmag": 2.0},
}


def _run(cfg):
    env = dict(os.environ, TORCHDYNAMO_DISABLE="1", MAGIC_DEVICE="cpu", CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, "-c", WORKER, REF_SRC, ROOT, json.dumps(cfg),
                        json.dumps(RECIPE_SHT + OTHER_SHT)],
                       capture_output=True, text=True, env=env, cwd="/tmp", timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):])


@pytest.fixture(scope="module", params=sorted(CONFIGS))
def glue(request):
    return request.param, _run(CONFIGS[request.param])


def test_recipe_names_and_positional_parameters(glue):
    _, out = glue
    for name, (ref_pos, ours) in out["sig"].items():
        assert ref_pos != "missing", (name, ours)
        assert ours[:len(ref_pos)] == ref_pos, (name, ref_pos, ours)


def test_configure_from_reference_copies_sizes_and_factors(glue):
    which, out = glue
    for k, (ref, ours) in out["cfg"].items():
        assert ours == ref, (k, ref, ours)
    if which == "anel":
        # the anelastic configuration has a nonzero dissipation number, so the
        # viscous/ohmic heating factors get_nl_anel reads are not the defaults
        assert out["cfg"]["ViscHeatFac"][0] != 0.0


def test_configure_from_reference_copies_radial_profiles(glue):
    _, out = glue
    bad = [k for k, ok in out["prof"].items() if not ok]
    assert not bad, bad
