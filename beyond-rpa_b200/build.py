"""Build librpa_b200.so in-tree for sm_100a.

    python beyond-rpa_b200/build.py [--verbose-ptxas]

nvcc cross-compiles without a GPU; the shared library is written next to this
file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB = HERE / "librpa_b200.so"
SOURCES = ["capi.cu", "scale_split.cu", "syrk_tc.cu", "dsyrk_f64.cu", "logdet.cu", "freq_grid.cu", "noalloc.cu", "gemm_f64.cu", "t2_kernels.cu", "sosex.cu", "sosex_tc.cu", "syevd.cu", "selftest.cu", "ozaki.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    deps.append(CSRC / "librpa_b200.map")
    deps.append(Path(__file__))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    if not force and not needs_build():
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden", "--expt-relaxed-constexpr",
                    f"-I{INCLUDE}", f"-I{CSRC}"]
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    procs = []
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        objs.append(obj)
        cmd = [nvcc(), *flags, "-c", str(src), "-o", str(obj)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if out.strip():
            sys.stderr.write(out)
        if p.returncode != 0:
            failed = True
            sys.stderr.write("FAILED: " + " ".join(cmd) + "\n")
    if failed:
        raise RuntimeError("nvcc compilation failed")
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc(), *ARCH, "-shared", "-Xlinker", "--no-undefined", "-Xlinker", f"--version-script={CSRC / 'librpa_b200.map'}",
            "-o", str(tmp), *map(str, objs)]
    subprocess.run(link, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=True if a.verbose_ptxas else a.force, verbose_ptxas=a.verbose_ptxas))
