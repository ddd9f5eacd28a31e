"""Build the sm_100a shared library ``vtp/libvtp.so`` from ``csrc/`` with nvcc, and
the C++ host interface ``vtp/libvtp_host.so`` (``host/``, the reference's Solver /
Object / SolverManager classes over the C ABI) with g++.

Usage: ``python build.py [--jobs N] [--force]``.  Objects go to ``_build/``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
OUT = HERE / "vtp" / "libvtp.so"
# Checked build (python build.py --checked): -DVTP_CHECKED adds device-side bounds checks of
# every neighbour-list entry and cell-segment slot (status bit VTP_ERR_BOUNDS instead of an
# out-of-range access); select it with VTP_LIBRARY=checked.
BUILD_CHECKED = HERE / "_build_checked"
OUT_CHECKED = HERE / "vtp" / "libvtp_checked.so"
HOST_OUT = HERE / "vtp" / "libvtp_host.so"
HOST = HERE / "host"
ROOT = HERE.parent

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def json_include() -> str:
    """Directory holding nlohmann/json.hpp (header-only JSON library shipped in the image)."""
    cands = []
    try:
        import sysconfig
        sp = Path(sysconfig.get_paths()["purelib"])
        cands.append(sp / "include" / "cudnn_frontend" / "thirdparty")
    except Exception:
        pass
    cands += [Path("/usr/include"), Path("/usr/local/include")]
    for c in cands:
        if (c / "nlohmann" / "json.hpp").exists():
            return str(c)
    raise RuntimeError("nlohmann/json.hpp not found")


def flags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                   "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", json_include(),
                   "-DVTP_BUILD"]


def compile_one(src: Path, force: bool, checked: bool = False) -> Path:
    obj = (BUILD_CHECKED if checked else BUILD) / (src.stem + ".o")
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "vtp.h"]
    if not force and obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc()] + flags() + (["-DVTP_CHECKED"] if checked else []) + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build_library(force: bool = False, jobs: int | None = None, checked: bool = False) -> Path:
    out = OUT_CHECKED if checked else OUT
    (BUILD_CHECKED if checked else BUILD).mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, checked), srcs))
    if force or not out.exists() or any(o.stat().st_mtime > out.stat().st_mtime for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(out)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return out


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, checked: bool = True) -> Path:
    """libvtp.so, the host interface, and (unless checked=False) the checked build."""
    build_library(force, jobs)
    if checked:
        build_library(force, jobs, checked=True)
    build_host(force)
    if verbose:
        print(f"built {OUT}")
    return OUT


def host_flags() -> list[str]:
    return ["-std=c++17", "-O2", "-fPIC", "-I", str(HOST / "include"), "-I", str(ROOT / "include"),
            "-I", json_include()]


def build_host(force: bool = False) -> Path:
    """libvtp_host.so: the C++ Solver/Object classes, linked against libvtp.so."""
    srcs = sorted((HOST / "src").glob("*.cpp"))
    deps = srcs + list((HOST / "include").rglob("*.hpp")) + [ROOT / "include" / "vtp.h", OUT]
    if not force and HOST_OUT.exists() and all(HOST_OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return HOST_OUT
    cmd = ["g++"] + host_flags() + ["-shared", "-o", str(HOST_OUT)] + [str(s) for s in srcs] + \
          ["-L", str(OUT.parent), "-lvtp", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host library build failed:\n{r.stdout}\n{r.stderr}")
    return HOST_OUT


def build_host_program(src: Path, out: Path) -> Path:
    """Compile a C++ program against the host interface (used by the example and its tests)."""
    cmd = ["g++"] + host_flags() + ["-o", str(out), str(src), "-L", str(HOST_OUT.parent), "-lvtp_host", "-lvtp",
                                    f"-Wl,-rpath,{HOST_OUT.parent}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"program build failed:\n{r.stdout}\n{r.stderr}")
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--no-checked", action="store_true", help="skip the checked build (libvtp_checked.so)")
    a = ap.parse_args()
    try:
        build(force=a.force, jobs=a.jobs, verbose=True, checked=not a.no_checked)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
