"""Build the in-tree CUDA library ``nsrno_b200/libnsrno_b200.so`` for sm_100a.

``python -m nsrno_b200.build`` (or ``build()``) runs nvcc on every ``.cu`` file of
``nsrno_b200/csrc`` and links them into one shared library with a plain C ABI
(``include/nsrno_b200.h``).  The CUDA runtime is linked statically, the way the
reference builds its native kernels (nsrno/native_time.py:32-33).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIBRARY = PACKAGE / "libnsrno_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found: the nsrno_b200 CUDA library cannot be built")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale():
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = list(sources()) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(p.stat().st_mtime > built for p in inputs)


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it; return its path."""
    if not force and not _stale():
        return LIBRARY
    nvcc = _nvcc()
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--extended-lambda",
                     f"-I{ROOT / 'include'}", f"-I{CSRC}"]
    jobs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *common, "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        jobs.append((cmd, str(obj)))
    # one nvcc per translation unit, side by side
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as pool:
        for done in [pool.submit(subprocess.run, cmd, check=True) for cmd, _ in jobs]:
            done.result()
    objects = [obj for _, obj in jobs]
    tmp = LIBRARY.with_suffix(".so.tmp")
    subprocess.run([nvcc, *ARCH, "-shared", "-o", str(tmp), *objects], check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
