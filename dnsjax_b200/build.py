"""Build libdnsb.so in-tree for sm_100a (``python -m dnsjax_b200.build``)."""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libdnsb.so"
SOURCES = ["passes.cu", "solver.cu", "imm.cu", "imm_batch.cu", "noalloc.cu", "precompute.cu",
           "learned.cu", "mlp_tc.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def needs_build(out: Path = OUT) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh"))
    deps.append(HERE.parent / "include" / "dnsb.h")
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source to an object in parallel (the translation units
    share no device symbols), then link the shared library."""
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    if not force and not needs_build():
        return OUT
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    with tempfile.TemporaryDirectory(prefix="dnsb_build_") as tmpdir:
        objs = [Path(tmpdir) / (Path(s).stem + ".o") for s in SOURCES]

        def compile_one(k):
            subprocess.run([nvcc(), *flags, "-c", str(CSRC / SOURCES[k]), "-o",
                            str(objs[k])], check=True)

        workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
        with ThreadPoolExecutor(max_workers=workers) as pool:
            list(pool.map(compile_one, range(len(SOURCES))))
        tmp = OUT.with_suffix(".so.tmp")
        subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp),
                        *[str(o) for o in objs]], check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
