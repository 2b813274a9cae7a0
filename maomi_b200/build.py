"""Build the CUDA library in-tree: ``maomi_b200/libmaomi_b200.so`` for sm_100a.

    python -m maomi_b200.build          # or maomi_b200.build.build()
"""

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
LIB = HERE / "libmaomi_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(SRC.glob("*.cu"))


def build(verbose=False, force=False):
    """Compile every ``csrc/*.cu`` into one shared library (parallel objects)."""
    srcs = sources()
    newest = max(p.stat().st_mtime for p in srcs + sorted(SRC.glob("*.cuh")) + [HERE.parent / "include" / "maomi_b200.h"])
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    obj_dir = HERE / "_build"
    obj_dir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    procs = []
    for src in srcs:
        obj = obj_dir / (src.stem + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, "-I", str(HERE.parent / "include"), "-c", str(src), "-o", str(obj)]
        procs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    objs = []
    failed = []
    for src, obj, proc in procs:
        out, _ = proc.communicate()
        if verbose and out:
            sys.stdout.write(out)
        if proc.returncode:
            failed.append((src.name, out))
        objs.append(str(obj))
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(f"{n}:\n{o}" for n, o in failed))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart_static" if False else "-cudart=static"]
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode:
        raise RuntimeError("link failed:\n" + res.stdout)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
