"""Place the reference's pure-Python packages of the Fourier-slice path in
``baseline/_ref`` (git-ignored) so that ``bench.py`` can time the unmodified
reference on the GPU.

``pip install --no-index --target baseline/_ref`` cannot build these packages
offline: their build backend (hatchling + hatch-vcs) is not installed.  The
packages are plain Python, so this recipe does what the install would do for
them: it copies each package's ``src`` tree into ``baseline/_ref``.  Run it
where the reference checkout exists, giving its root as the argument or in
``TT_REFERENCE_ROOT``:

    python baseline/install_reference.py /path/to/reference
"""

from __future__ import annotations

import os
import shutil
import sys

PACKAGES = ("torch-fourier-slice", "torch-image-interpolation", "torch-grid-utils", "torch-ctf")


def main() -> int:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TT_REFERENCE_ROOT")
    if not ref:
        print("usage: install_reference.py REFERENCE_ROOT (or set TT_REFERENCE_ROOT)", file=sys.stderr)
        return 2
    dest = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")
    os.makedirs(dest, exist_ok=True)
    for pkg in PACKAGES:
        src = os.path.join(ref, "packages", "primitives", pkg, "src")
        for name in os.listdir(src):
            if name.endswith(".egg-info") or name.startswith("."):
                continue
            target = os.path.join(dest, name)
            if os.path.exists(target):
                shutil.rmtree(target)
            shutil.copytree(os.path.join(src, name), target,
                            ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    print(f"reference packages in {dest}: {sorted(os.listdir(dest))}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
