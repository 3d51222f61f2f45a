"""Build the sm_100a shared library ``libtfb200.so`` in-tree with nvcc.

``python -m deep_frame_b200.build`` compiles every ``csrc/*.cu`` translation
unit for ``sm_100a`` (in parallel) and links them into
``deep_frame_b200/libtfb200.so`` with a statically linked CUDA runtime, so
the library has no runtime dependency beyond the driver.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
INCLUDE = ROOT / "include"
LIBRARY = PACKAGE / "libtfb200.so"
BUILD = ROOT / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc():
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libtfb200.so")
    return found


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale(objects):
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > built for p in inputs)


def build(force=False, verbose=False):
    """Compile and link the library; returns its path.  Raises on any compiler error."""
    srcs = sources()
    BUILD.mkdir(exist_ok=True)
    objects = [BUILD / (s.stem + ".o") for s in srcs]
    if not force and not _stale(objects):
        return LIBRARY
    compiler = nvcc()

    def compile_one(pair):
        src, obj = pair
        cmd = [compiler, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        run = subprocess.run(cmd, capture_output=True, text=True)
        if run.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{run.stderr}")
        if verbose and run.stderr:
            sys.stderr.write(run.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        list(pool.map(compile_one, zip(srcs, objects)))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [compiler, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objects)]
    run = subprocess.run(cmd, capture_output=True, text=True)
    if run.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{run.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
