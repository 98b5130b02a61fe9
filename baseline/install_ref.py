"""Install the reference package (torch-sim-atomistic) into ``baseline/_ref``.

The stock offline command

    python -m pip install --no-index --no-build-isolation \
        --find-links /opt/wheelhouse --target baseline/_ref /root/reference

fails in this image: the reference's ``[build-system]`` names ``uv_build``, which
is not in the offline wheelhouse.  The reference is pure Python, so this script
copies the source tree to a temporary directory, replaces only the
``[build-system]`` table of the copy's ``pyproject.toml`` by setuptools (with a
package filter for ``torch_sim``), and installs that copy with the same pip
flags plus ``--no-deps`` (``h5py``, ``tables`` and ``nvalchemi-toolkit-ops`` are
not in the wheelhouse).  The installed ``torch_sim`` tree is then compared file
by file with the source: the package code is the reference's, unmodified.

Usage: ``python baseline/install_ref.py [/path/to/reference]``.  Does nothing
when the reference tree is absent (the GPU box has none; the installed copy
travels with the repository instead).
"""

from __future__ import annotations

import filecmp
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
TARGET = os.path.join(HERE, "_ref")

_OLD_BUILD = '''[build-system]
requires = ["uv_build>=0.7.12"]
build-backend = "uv_build"
'''
_NEW_BUILD = '''[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"

[tool.setuptools.packages.find]
include = ["torch_sim*"]
'''


def _same_tree(a: str, b: str) -> bool:
    """Every .py file under a exists in b with the same bytes."""
    for root, _, files in os.walk(a):
        for f in files:
            if not f.endswith(".py"):
                continue
            pa = os.path.join(root, f)
            pb = os.path.join(b, os.path.relpath(pa, a))
            if not os.path.exists(pb) or not filecmp.cmp(pa, pb, shallow=False):
                return False
    return True


def installed() -> bool:
    return os.path.isdir(os.path.join(TARGET, "torch_sim"))


def install(ref_root: str = "/root/reference", verbose: bool = False) -> bool:
    """Install the reference into baseline/_ref; True if it is there afterwards.
    An existing install is kept only while it matches the source tree."""
    src_pkg = os.path.join(ref_root, "torch_sim")
    if not os.path.isdir(src_pkg):
        return installed()
    if installed():
        dst_pkg = os.path.join(TARGET, "torch_sim")
        if _same_tree(src_pkg, dst_pkg) and _same_tree(dst_pkg, src_pkg):
            return True
        shutil.rmtree(TARGET)
    with tempfile.TemporaryDirectory(prefix="tsref_src_") as tmp:
        src = os.path.join(tmp, "torch-sim")
        os.makedirs(src)
        shutil.copytree(os.path.join(ref_root, "torch_sim"), os.path.join(src, "torch_sim"),
                        ignore=shutil.ignore_patterns("__pycache__"))
        for f in ("pyproject.toml", "README.md", "LICENSE"):
            if os.path.exists(os.path.join(ref_root, f)):
                shutil.copy(os.path.join(ref_root, f), os.path.join(src, f))
        pp = os.path.join(src, "pyproject.toml")
        text = open(pp).read()
        if _OLD_BUILD not in text:
            raise RuntimeError("unexpected [build-system] table in the reference pyproject.toml")
        with open(pp, "w") as fh:
            fh.write(text.replace(_OLD_BUILD, _NEW_BUILD))
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
               "--no-deps", "--find-links", "/opt/wheelhouse", "--target", TARGET, src]
        r = subprocess.run(cmd, capture_output=not verbose, text=True)
        if r.returncode != 0:
            if not verbose:
                sys.stderr.write((r.stdout or "")[-2000:] + (r.stderr or "")[-2000:])
            return False
    if not _same_tree(os.path.join(ref_root, "torch_sim"), os.path.join(TARGET, "torch_sim")):
        shutil.rmtree(TARGET, ignore_errors=True)
        raise RuntimeError("installed torch_sim differs from the reference source tree")
    return True


if __name__ == "__main__":
    ok = install(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", verbose=True)
    print("baseline/_ref:", "installed" if ok else "not installed")
