"""Build libvamcore.so (all CUDA sources of the package) for sm_100a.

    python -m vamtoolbox_b200.csrc.build [--force] [--verbose-ptxas]

Each .cu file is compiled to an object with nvcc in parallel, then linked into
vamtoolbox_b200/libvamcore.so next to the package, so the library travels
with the source tree.  Objects go to vamtoolbox_b200/_build/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent
ROOT = PKG.parent
OUT = PKG / "libvamcore.so"
OBJ = PKG / "_build"
SOURCES = ["capi.cu", "parallel.cu", "optim.cu", "raytrace.cu", "output.cu", "vecgeom.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (set NVCC or put /usr/local/cuda/bin on PATH)")


def _flags(verbose_ptxas: bool):
    f = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
         "-I", str(ROOT / "include"), "--expt-relaxed-constexpr"]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def _inputs():
    deps = [CSRC / s for s in SOURCES] + [CSRC / "vam_internal.cuh", ROOT / "include" / "vam.h"]
    deps += list(CSRC.glob("*.cuh"))
    return deps


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _inputs() if p.exists())


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    if not force and up_to_date():
        return OUT
    OBJ.mkdir(exist_ok=True)
    cc = nvcc()
    flags = _flags(verbose_ptxas)

    def compile_one(src):
        obj = OBJ / (Path(src).stem + ".o")
        cmd = [cc, *flags, "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose_ptxas:
        for _, err in results:
            sys.stderr.write(err)
    objs = [str(o) for o, _ in results]
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    args = ap.parse_args()
    p = build(force=args.force, verbose_ptxas=args.verbose_ptxas)
    print(p)


if __name__ == "__main__":
    main()
