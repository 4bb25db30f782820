"""Install the unmodified reference (deltaMic 0.1.0) into ``baseline/_ref``.

    python baseline/install_reference.py [<reference checkout>]

The reference's ``setup.py`` calls ``torch.cuda.is_available()`` without importing
``torch`` (setup.py:39), so ``pip install`` of the checkout stops with
``NameError: name 'torch' is not defined`` before it builds anything.  This recipe
runs that same ``setup.py``, unchanged, from a copy under a temporary directory
with ``torch`` already imported into its globals, builds the wheel it describes
(without a GPU in the build container: the pure-Python package, the branch of
setup.py that builds no CUDA extension), and installs that wheel with pip into
``baseline/_ref`` (``--no-deps``: largesteps, robust_laplacian and trimesh are
absent offline; the CPU render path ``deltamic.render`` / ``deltamic.psf`` does
not import them).  No reference source is edited and nothing is written to the
checkout.  ``bench.py --impl reference`` imports ``deltamic.render.MeshFTPy`` from
there.
"""
from __future__ import annotations

import os
import runpy
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
TARGET = os.path.join(HERE, "_ref")


def main(src: str) -> None:
    if not os.path.isfile(os.path.join(src, "setup.py")):
        raise SystemExit(f"no setup.py under {src}")
    import torch  # noqa: F401  (supplied to setup.py's globals)
    with tempfile.TemporaryDirectory() as tmp:
        work = os.path.join(tmp, "deltamic")
        shutil.copytree(src, work, ignore=shutil.ignore_patterns(".git", "*.pyc", "__pycache__"))
        dist = os.path.join(tmp, "dist")
        cwd = os.getcwd()
        argv = sys.argv
        try:
            os.chdir(work)
            sys.argv = ["setup.py", "-q", "bdist_wheel", "-d", dist]
            runpy.run_path("setup.py", init_globals={"torch": torch}, run_name="__main__")
        finally:
            os.chdir(cwd)
            sys.argv = argv
        wheels = [os.path.join(dist, w) for w in os.listdir(dist) if w.endswith(".whl")]
        if len(wheels) != 1:
            raise SystemExit(f"expected one wheel, found {wheels}")
        if os.path.isdir(TARGET):
            shutil.rmtree(TARGET)
        subprocess.run([sys.executable, "-m", "pip", "install", "--no-index", "--no-deps",
                        "--no-build-isolation", "--target", TARGET, wheels[0]], check=True)
    print("installed", TARGET)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DELTAMIC_REF", ""))
