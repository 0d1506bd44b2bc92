"""Build liblitho_b200.so for sm_100a with nvcc.

    python lithobat_b200/csrc/build.py [--force] [--verbose-ptxas]

Every .cu in this folder is compiled for sm_100a only (no PTX, no other
arch) into lithobat_b200/_build/*.o and linked into lithobat_b200/liblitho_b200.so,
next to the package so it ships with the source tree. Rebuilds only what
changed (by mtime of the .cu and every header).
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
OUT = PKG / "liblitho_b200.so"
BUILD = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def flags(verbose_ptxas: bool) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = False) -> Path:
    subprocess.run([sys.executable, str(CSRC / "gen_twiddles.py"), str(CSRC / "twiddles.cuh")],
                   check=True)
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hmt = headers_mtime()
    cc = nvcc()
    jobs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        if force or verbose_ptxas or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hmt):
            jobs.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [cc, *flags(verbose_ptxas), "-c", str(s), "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for s, r in ex.map(compile_one, jobs):
                if r.returncode != 0:
                    sys.stderr.write(r.stdout + r.stderr)
                    raise RuntimeError(f"nvcc failed on {s.name}")
                if (verbose_ptxas or r.stderr.strip()) and not quiet:
                    sys.stderr.write(f"--- {s.name}\n{r.stderr}")
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    orphans = [o for o in BUILD.glob("*.o") if o not in objs]   # objects of removed sources
    for o in orphans:
        o.unlink()
    if jobs or orphans or not OUT.exists() or OUT.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [cc, *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of liblitho_b200.so failed")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
