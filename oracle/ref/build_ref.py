"""Build the reference's own solvers from their sources into ``oracle/_ref/libvtref.so``.

Recipe (test infrastructure): nvcc compiles the reference's UGNS, PBF, DFSPH,
IMM and IMM-CT sources plus the framework / JSON / model files they need,
exactly as they lie under the reference tree, for sm_100a with
``-O3 -DNDEBUG``, together with this directory's shims (``shim/``) and the
harness ``ref_harness.cu``.  Nothing is written outside ``oracle/_ref/``.
The reference's own CMake build is not used (it needs vcpkg and MSVC-only
flags).  ``CommonFunc.cpp`` is left out: the harness supplies ``cal_mean``.

Builds without a GPU (nvcc cross-compiles for sm_100a); the library is loaded where the
golden fixtures are generated.  The reference checkout is given by the environment
variable VTP_REFERENCE, the ``reference`` argument of ``build``/``available`` or
``--reference PATH`` on the command line; there is no default location.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE.parent / "_ref"


def reference_root(reference: str | os.PathLike | None = None) -> Path | None:
    """The reference checkout: the argument, else VTP_REFERENCE, else none."""
    p = reference or os.environ.get("VTP_REFERENCE")
    return Path(p) if p else None

SOURCES = [
    "Runtime/Source/Framework/Object.cpp",
    "Runtime/Source/Framework/ObjectComponents.cpp",
    "Runtime/Source/Framework/Solver.cpp",
    "Runtime/Source/Modules/NeighborSearch/UGNS/UniformGridNeighborSearch.cpp",
    "Runtime/Source/Modules/NeighborSearch/UGNS/UGNSCudaImpl.cu",
    "Runtime/Source/Solvers/PBF/PBFSolver.cpp",
    "Runtime/Source/Solvers/PBF/PBFCudaImpl.cu",
    "Runtime/Source/Solvers/DFSPH/DFSPHSolver.cpp",
    "Runtime/Source/Solvers/DFSPH/DFSPHCudaImpl.cu",
    "Runtime/Source/Solvers/IMM/IMMSolver.cpp",
    "Runtime/Source/Solvers/IMM/IMMCudaImpl.cu",
    "Runtime/Source/Solvers/IMM-CT/IMMCTSolver.cpp",
    "Runtime/Source/Solvers/IMM-CT/IMMCTCudaImpl.cu",
    "Library/Source/JSON/JSONHandler.cpp",
    "Library/Source/Model/ModelHandler.cpp",
    "Library/Source/Model/ExportUtil.cpp",
]


def json_include() -> str:
    import sysconfig
    c = Path(sysconfig.get_paths()["purelib"]) / "include" / "cudnn_frontend" / "thirdparty"
    if (c / "nlohmann" / "json.hpp").exists():
        return str(c)
    raise RuntimeError("nlohmann/json.hpp not found")


def available(reference: str | os.PathLike | None = None) -> bool:
    ref = reference_root(reference)
    return ref is not None and (ref / "Simulator").exists()


def build(force: bool = False, reference: str | os.PathLike | None = None) -> Path:
    out = OUT_DIR / "libvtref.so"
    if not available(reference):
        if out.exists():
            return out
        raise RuntimeError(f"reference sources not found (VTP_REFERENCE / --reference: {reference_root(reference)})")
    REF = reference_root(reference)
    SIM = REF / "Simulator"
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    gen = OUT_DIR / "gen" / "ConfigTemplates"
    gen.mkdir(parents=True, exist_ok=True)
    cfg_dir = OUT_DIR / "ConfigTemplates"
    if (REF / "ConfigTemplates").exists():
        shutil.copytree(REF / "ConfigTemplates", cfg_dir, dirs_exist_ok=True)
    (gen / "RealPath.h").write_text(
        "#pragma once\n"
        f'#define VP_SRC_DIR "{REF}/"\n'
        f'#define VP_CONFIG_DIR "{cfg_dir}/"\n'
        f'#define VP_EXAMPLES_DIR "{REF}/Examples/"\n')
    incs = ["-I", str(SIM / "Runtime" / "Include"), "-I", str(SIM / "Library" / "Include"),
            "-I", str(HERE / "shim"), "-I", str(OUT_DIR / "gen"), "-I", json_include()]
    flags = ["-O3", "-DNDEBUG", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
             "-include", str(HERE / "shim" / "vp_compat.h"), "-w"] + incs
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    jobs = []
    for rel in SOURCES:
        src = SIM / rel
        jobs.append((src, obj_dir / (rel.replace("/", "_") + ".o")))
    jobs.append((HERE / "ref_harness.cu", obj_dir / "ref_harness.o"))

    def one(job):
        src, obj = job
        if not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime:
            return obj
        lang = ["-x", "cu"] if src.suffix == ".cu" else ["-x", "c++"]
        r = subprocess.run([nvcc] + flags + lang + ["-c", str(src), "-o", str(obj)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{src}:\n{r.stderr[-4000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(one, jobs))
    r = subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(out)] +
                       [str(o) for o in objs] + ["-lcudart"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return out


if __name__ == "__main__":
    ref = sys.argv[sys.argv.index("--reference") + 1] if "--reference" in sys.argv else None
    try:
        print(build(force="--force" in sys.argv, reference=ref))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
