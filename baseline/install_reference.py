"""Install the unchanged reference modules into ``baseline/_ref/`` (git-ignored).

    python baseline/install_reference.py --source <reference checkout>

The reference is a flat directory of Python modules (config.py, physics.py,
solver.py, main.py) with no packaging metadata, so ``pip install <dir>``
refuses it ("Neither 'setup.py' nor 'pyproject.toml' found").  This recipe
copies the checkout to a temporary directory, adds a minimal pyproject.toml
naming the four modules (no dependencies: CuPy and matplotlib are supplied
by the stand-ins in this directory at run time) and runs

    python -m pip install --no-index --no-build-isolation --no-deps \
        --find-links /opt/wheelhouse --target baseline/_ref <copy>

The module sources are not edited.  ``baseline/_ref/SOURCE.json`` records the
SHA-256 of each installed module next to the checkout's, so a run can show
that it executes the reference as published.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
DEST = os.path.join(HERE, "_ref")
MODULES = ("config", "physics", "solver", "main")

PYPROJECT = """[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"

[project]
name = "aeromhd-reference"
version = "0.0.0"
description = "AeroMHD-CUDA reference modules, installed unchanged"

[tool.setuptools]
py-modules = [%s]
"""


def sha256(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def install(source: str, dest: str = DEST) -> dict:
    missing = [m for m in MODULES if not os.path.isfile(os.path.join(source, m + ".py"))]
    if missing:
        raise FileNotFoundError(f"{source} lacks the reference modules {missing}")
    with tempfile.TemporaryDirectory(prefix="amhd_ref_pkg_") as tmp:
        for m in MODULES:
            shutil.copy2(os.path.join(source, m + ".py"), os.path.join(tmp, m + ".py"))
        with open(os.path.join(tmp, "pyproject.toml"), "w") as f:
            f.write(PYPROJECT % ", ".join(f'"{m}"' for m in MODULES))
        if os.path.isdir(dest):
            shutil.rmtree(dest)
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation", "--no-deps",
               "--find-links", "/opt/wheelhouse", "--target", dest, tmp]
        subprocess.check_call(cmd)
    record = {"source_sha256": {m: sha256(os.path.join(source, m + ".py")) for m in MODULES},
              "installed_sha256": {m: sha256(os.path.join(dest, m + ".py")) for m in MODULES},
              "pip": " ".join(cmd[1:-1]) + " <copy of the checkout>"}
    record["unchanged"] = record["source_sha256"] == record["installed_sha256"]
    with open(os.path.join(dest, "SOURCE.json"), "w") as f:
        json.dump(record, f, indent=1)
    return record


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--source", default=os.environ.get("AMHD_REFERENCE_DIR"),
                    help="reference checkout (default: $AMHD_REFERENCE_DIR)")
    ap.add_argument("--dest", default=DEST)
    a = ap.parse_args(argv)
    if not a.source:
        ap.error("give --source or set AMHD_REFERENCE_DIR")
    rec = install(a.source, a.dest)
    print(json.dumps({"dest": a.dest, "unchanged": rec["unchanged"]}))
    return 0 if rec["unchanged"] else 1


if __name__ == "__main__":
    sys.exit(main())
