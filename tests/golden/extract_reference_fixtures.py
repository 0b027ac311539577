"""Extract the reference's own tiny fixtures and known answers into JSON.

Reads (text only, nothing is executed):
  tests/helpers.rs:37-63   make_tiny_train  (20 users x 10 items, 56 ratings)
  tests/helpers.rs:69-95   make_tiny_probe  (20 ratings)
  tests/regressors_test.rs:28-73  the shared regression-test config
  tests/regressors_test.rs:75-93  tsvdx4 probe RMSE known answer
  tests/regressors_test.rs:157-175 tsvdx4p probe RMSE known answer
Run from the repo root:  python tests/golden/extract_reference_fixtures.py REF_ROOT
(REF_ROOT: a checkout of the reference repository).
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: extract_reference_fixtures.py REF_ROOT")
ref = sys.argv[1]
helpers = open(os.path.join(ref, "tests/helpers.rs")).read()
regs = open(os.path.join(ref, "tests/regressors_test.rs")).read()


def table(fn_name):
    body = helpers.split(f"pub fn {fn_name}()")[1].split("build_dataset(")[0]
    rows = re.findall(r"\(\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\)", body)
    return [[int(a), int(b), int(c), int(d)] for a, b, c, d in rows]


def known_rmse(test_name):
    body = regs.split(f"fn {test_name}()")[1].split("#[test]")[0]
    return float(re.search(r"assert!\(rmse == ([0-9.]+)\)", body).group(1))


cfg_body = regs.split("macro_rules! cfg")[1].split("$($extra)*")[0]
cfg = {}
for k, v in re.findall(r"(\w+):\s*([-0-9.e]+|true|false),", cfg_body):
    cfg[k] = v == "true" if v in ("true", "false") else float(v)

out = {
    "source": "reference tests/helpers.rs and tests/regressors_test.rs",
    "tiny_train": table("make_tiny_train"),
    "tiny_probe": table("make_tiny_probe"),
    "n_users": 20,
    "n_items": 10,
    "regression_cfg": cfg,
    "tsvdx4_probe_rmse": known_rmse("tsvdx4_probe_rmse_regression"),
    "tsvdx4p_probe_rmse": known_rmse("tsvdx4p_probe_rmse_regression"),
}
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "reference_fixtures.json"), "w") as f:
    json.dump(out, f, indent=1)
print(len(out["tiny_train"]), len(out["tiny_probe"]), out["tsvdx4_probe_rmse"], out["tsvdx4p_probe_rmse"])
print(cfg)
