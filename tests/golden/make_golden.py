"""Regenerate tests/golden/ref_helpers.json from the reference's own CPU helpers.

Builds oracle/ref_helpers (which compiles 3D_elastic_RTM/zzzzz and
3D_elastic_RTM/3D_zzzzz from the reference tree) into oracle/_ref/ref_helpers,
runs it and stores its JSON output.  Needs the reference tree; the committed
fixture is what the tests read.

    python tests/golden/make_golden.py [--ref /root/reference]
"""
import argparse
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

ap = argparse.ArgumentParser()
ap.add_argument("--ref", default="/root/reference")
args = ap.parse_args()
subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle", "ref_helpers"), f"REF={args.ref}"],
               check=True)
out = subprocess.run([os.path.join(REPO, "oracle", "_ref", "ref_helpers")], check=True,
                     capture_output=True, text=True).stdout
data = json.loads(out)
data["_about"] = ("Outputs of the reference's own CPU helpers (make_ricker_new, "
                  "make_coe_optimized_new, make_attenuation_new, coe_attenuation_3d_new2, "
                  "add_pml_layers_v_h, vp_set_vs, vp_set_density, cpu_laplace, suhilbt) on the "
                  "fixed inputs in "
                  "oracle/ref_helpers/ref_helpers.cpp; generated by tests/golden/make_golden.py")
with open(os.path.join(HERE, "ref_helpers.json"), "w") as f:
    json.dump(data, f, indent=0)
print("wrote", os.path.join(HERE, "ref_helpers.json"), sorted(data))
