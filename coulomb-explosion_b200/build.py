"""Build recipe for libce_gpu.so (sm_100a) and the C++ drop-in (coulomb::gpu).

Compiles every CUDA translation unit with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` in parallel
into ``_build/`` and links the shared library in-tree (next to this file), so
it travels with the repository snapshot. Incremental by default (a unit is
rebuilt only when a source or header is newer than its object); `force=True`,
which __graft_entry__.build() passes, recompiles everything.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = ROOT / "include"
LIB = PKG / "libce_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ftz=true", "-Xcompiler", "-fPIC",
                  "-I", str(INCLUDE), "-I", str(CSRC)]

# (object name, source, extra flags)
UNITS = [("ce_gpu.o", "ce_gpu.cu", []), ("probe.o", "probe.cu", []), ("noalloc.o", "noalloc.cu", []),
         ("mixed.o", "mixed.cu", []), ("sampler.o", "sampler.cu", ["-Xcompiler", "-ffp-contract=off"]),
         ("mlp.o", "mlp.cu", []), ("closure.o", "closure.cu", []), ("verlet.o", "verlet.cu", [])] + [
    (f"kernels_fixed_m{m}.o", "kernels_fixed.cu", [f"-DCE_MODE={m}"]) for m in range(4)
] + [(f"kernels_atom_m{m}.o", "kernels_atom.cu", [f"-DCE_MODE={m}"]) for m in range(4)]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return (list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.h"))
            + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_headers(), Path(__file__)])


def build_cuda(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    jobs = []
    for obj, src, extra in UNITS:
        o, s = BUILD / obj, CSRC / src
        if force or _stale(o, s) or ptxas_info:
            cmd = [nvcc, *NVFLAGS, *extra, "-c", str(s), "-o", str(o)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append((obj, cmd))

    def run(job):
        obj, cmd = job
        p = subprocess.run(cmd, capture_output=True, text=True)
        return obj, p

    failed = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for obj, p in ex.map(run, jobs):
            if verbose or ptxas_info:
                sys.stderr.write(p.stdout + p.stderr)
            if p.returncode != 0:
                failed.append((obj, p.stderr))
    if failed:
        msg = "\n".join(f"--- {o}\n{e}" for o, e in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    objs = [str(BUILD / o) for o, _, _ in UNITS]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{p.stderr}")
    return LIB


HOST = PKG / "host"
BIN = PKG / "bin"
HOST_LIB = PKG / "libce_host.so"
CUDA_LIB = Path("/usr/local/cuda/lib64")


def _cxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def _run(cmd: list[str]) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{p.stderr}")


def reference_dir(explicit: str | os.PathLike | None = None) -> Path | None:
    """The reference checkout (its include/coulomb/ and src/) the host library is
    built beside: `explicit`, else $COULOMB_REFERENCE_DIR; None if neither names
    a checkout."""
    cand = explicit or os.environ.get("COULOMB_REFERENCE_DIR")
    if cand and (Path(cand) / "include" / "coulomb" / "driver.hpp").exists():
        return Path(cand)
    return None


ENGINE_LIB = BIN / "libcoulomb_engine.so"


def build_host(reference: str | os.PathLike | None = None, force: bool = False) -> bool:
    """The C++ drop-in, built beside the reference's coulomb::engine:

    * bin/libcoulomb_engine.so -- the reference's own engine library
      (src/system.cpp, integrators.cpp, driver.cpp, sampler.cpp, compiled where
      they lie with its Release flags, src/CMakeLists.txt:3-17), the host
      project the drop-in plugs into;
    * libce_host.so -- coulomb::gpu (BatchedRK45, run_to_convergence_batch,
      PhiloxBallSampler, DatasetWriter) compiled against the reference's
      include/coulomb headers and libce_gpu.so;
    * bin/ce_generate_dataset and bin/ce_test_host, linked against both.

    Needs a reference checkout (`reference_dir`); returns False and builds
    nothing without one."""
    ref = reference_dir(reference)
    if ref is None:
        print("build_host: no reference checkout (COULOMB_REFERENCE_DIR); C++ drop-in not built", file=sys.stderr)
        return False
    cxx = _cxx()
    ref_inc = ref / "include"
    inc = ["-I", str(HOST / "include"), "-I", str(ref_inc), "-I", str(INCLUDE)]
    flags = ["-std=c++20", "-O2", "-ffp-contract=off", "-Wall", "-Wextra"]
    BIN.mkdir(exist_ok=True)
    eng_srcs = [ref / "src" / f for f in ("system.cpp", "integrators.cpp", "driver.cpp", "sampler.cpp")]
    ref_hdrs = list((ref_inc / "coulomb").glob("*.hpp"))
    newest_eng = max(p.stat().st_mtime for p in [*eng_srcs, *ref_hdrs])
    if force or not ENGINE_LIB.exists() or ENGINE_LIB.stat().st_mtime < newest_eng:
        _run([cxx, "-std=c++20", "-O3", "-DNDEBUG", "-fPIC", "-shared", "-I", str(ref_inc), *map(str, eng_srcs),
              "-o", str(ENGINE_LIB)])
    srcs = sorted((HOST / "src").glob("*.cpp"))
    hdrs = list((HOST / "include").rglob("*.hpp")) + list(INCLUDE.glob("*.h")) + ref_hdrs
    newest_in = max(p.stat().st_mtime for p in [*srcs, *hdrs, LIB])
    if force or not HOST_LIB.exists() or HOST_LIB.stat().st_mtime < newest_in:
        _run([cxx, *flags, "-fPIC", "-shared", *inc, *map(str, srcs), "-L", str(PKG), "-lce_gpu",
              "-Wl,-rpath,$ORIGIN", "-o", str(HOST_LIB)])
    progs = {"ce_generate_dataset": HOST / "examples" / "generate_dataset.cpp",
             "ce_test_host": ROOT / "tests" / "cpp" / "test_host.cpp"}
    for name, src in progs.items():
        out = BIN / name
        if not force and out.exists() and out.stat().st_mtime >= max(
                src.stat().st_mtime, HOST_LIB.stat().st_mtime, ENGINE_LIB.stat().st_mtime):
            continue
        _run([cxx, *flags, *inc, "-I", "/usr/local/cuda/include", str(src), "-L", str(PKG), "-lce_host", "-lce_gpu",
              "-L", str(BIN), "-lcoulomb_engine", "-L", str(CUDA_LIB), "-lcudart", "-Wl,-rpath,$ORIGIN",
              "-Wl,-rpath,$ORIGIN/..", "-Wl,-rpath," + str(CUDA_LIB), "-o", str(out)])
    return True


def build_all(verbose: bool = False, reference: str | os.PathLike | None = None, force: bool = False) -> None:
    """Everything; `force` recompiles every unit whatever the timestamps say."""
    build_cuda(verbose=verbose, force=force)
    build_host(reference, force=force)


if __name__ == "__main__":
    build_cuda(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
