"""Builds the B200 G-MAPF shared library in-tree (gmapf_b200/libgmapf_b200.so)
and the CPU oracle (oracle/liboracle.so).

CUDA sources are compiled by nvcc for sm_100a only; host sources by g++.
Every translation unit uses -ffp-contract=off (host) and the kernels spell
their arithmetic with explicit round-to-nearest intrinsics, so results are
bit-identical to the oracle's IEEE binary32 evaluation.

The navmesh builder (FillMapEnd) is compiled against the CDT headers that
the reference project vendors; their include directory comes from
GMAPF_CDT_DIR.  Without it the library is built without FillMapEnd.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libgmapf_b200.so"
OBJ = PKG / "_build"
ORACLE_DIR = ROOT / "oracle"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["search.cu", "kernels.cu", "device.cu", "serve.cu", "noalloc.cu"]
CPP_SOURCES = ["hostmap.cpp", "capi.cpp"]
CDT_SOURCE = "navmesh_cdt.cpp"


# Where the reference project's source tree lies (build time only: its CDT
# headers are compiled into the navmesh builder, and its container headers
# into the oracle's pinning harness).  Nothing at run time reads it.
REF_DIR = os.environ.get("GMAPF_REF_DIR", "/root/reference")


def cdt_dir() -> str | None:
    d = os.environ.get("GMAPF_CDT_DIR") or os.path.join(REF_DIR, "include")
    if os.path.isfile(os.path.join(d, "CDT", "CDT.h")):
        return d
    return None


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _sources() -> list[Path]:
    return [CSRC / s for s in CU_SOURCES + CPP_SOURCES + [CDT_SOURCE]] + list(CSRC.glob("*.h")) + list(
        CSRC.glob("*.cuh")) + [ROOT / "include" / "gmapf_c.h", Path(__file__)]


def needs_build(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.exists() and p.stat().st_mtime > t for p in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build(OUT, _sources()):
        return OUT
    OBJ.mkdir(exist_ok=True)
    inc = ["-I", str(CSRC), "-I", str(ROOT / "include"), "-I", os.path.join(CUDA_HOME, "include")]
    jobs = []
    for s in CU_SOURCES:
        o = OBJ / (s + ".o")
        jobs.append([NVCC, "-c", str(CSRC / s), "-o", str(o), "-O3", "-std=c++17", *ARCH, "-lineinfo",
                     "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-O3", *inc])
    for s in CPP_SOURCES:
        o = OBJ / (s + ".o")
        jobs.append(["g++", "-c", str(CSRC / s), "-o", str(o), "-O2", "-std=c++17", "-fPIC",
                     "-ffp-contract=off", *inc])
    cdt = cdt_dir()
    o = OBJ / (CDT_SOURCE + ".o")
    cmd = ["g++", "-c", str(CSRC / CDT_SOURCE), "-o", str(o), "-O2", "-std=c++17", "-fPIC",
           "-ffp-contract=off", *inc]
    if cdt:
        cmd += ["-DGMAPF_HAVE_CDT", "-isystem", cdt]
    jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        list(ex.map(_run, jobs))
    objs = [str(OBJ / (s + ".o")) for s in CU_SOURCES + CPP_SOURCES + [CDT_SOURCE]]
    tmp = OUT.with_suffix(".so.tmp")
    _run([NVCC, "-shared", *ARCH, "-o", str(tmp), *objs, "-Xcompiler", "-fPIC", "-lpthread"])
    os.replace(tmp, OUT)
    if verbose:
        print(f"built {OUT} (CDT navmesh builder: {'yes' if cdt else 'no'})")
    return OUT


def build_oracle(force: bool = False) -> Path:
    out = ORACLE_DIR / "liboracle.so"
    deps = [ORACLE_DIR / "gmapf_oracle.cpp", ORACLE_DIR / "gmapf_oracle.h", ORACLE_DIR / "navmesh_oracle.cpp",
            ORACLE_DIR / "Makefile"]
    if force or needs_build(out, deps):
        cdt = cdt_dir()
        _run(["make", "-s", "-C", str(ORACLE_DIR), "-B" if force else "all"] + ([f"CDT_DIR={cdt}"] if cdt else []))
    return out


def ptxas_report() -> str:
    """Registers / spills / shared memory of the kernels (nvcc -Xptxas -v)."""
    lines = []
    for s in CU_SOURCES:
        r = subprocess.run([NVCC, "-c", str(CSRC / s), "-o", os.devnull, "-O3", "-std=c++17", *ARCH,
                            "-Xptxas", "-v", "-I", str(CSRC), "-I", str(ROOT / "include")],
                           capture_output=True, text=True)
        lines.append(r.stderr)
    return "\n".join(lines)


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_library(force=force, verbose=True)
    build_oracle(force=force)
    if "--ptxas" in sys.argv:
        print(ptxas_report())
