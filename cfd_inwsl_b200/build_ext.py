"""Build libcfdgpu.so (sm_100a) in-tree with nvcc.

    python -m cfd_inwsl_b200.build_ext [--jobs N] [--force]

The sweep kernels are instantiated per (flavour, NV, interpolator family):
  * flavour "strict": --fmad=false, reference operation order (bitwise parity);
  * flavour "fast":   FMA contraction plus the CFD_FAST algebraic rewrites.
Objects go to cfd_inwsl_b200/_build/, the library to cfd_inwsl_b200/libcfdgpu.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcfdgpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FAMILIES = [0, 1, 2, 3, 4, 5]
NVS = [3, 4, 5]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def common_flags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
                   "-I", str(CSRC)]


def units() -> list[tuple[Path, Path, list[str]]]:
    out = []
    headers = [CSRC / f for f in ("euler_math.cuh", "mixed.cuh", "sweep.cuh", "sweep_params.h")]
    for flavour in ("strict", "fast"):
        for nv in NVS:
            for fam in FAMILIES:
                obj = BUILD / f"sweep_{flavour}_nv{nv}_f{fam}.o"
                flags = ["-DCFD_NS=" + flavour, f"-DCFD_NV={nv}", f"-DCFD_FAM={fam}"]
                flags += ["--fmad=false"] if flavour == "strict" else ["--fmad=true", "-DCFD_FAST"]
                out.append((CSRC / "sweep_inst.cu", obj, flags, headers))
    out.append((CSRC / "api.cu", BUILD / "api.o", ["--fmad=false", "-DCFD_NS=api"],
                headers + [CSRC / "sweep_dispatch.h", CSRC / "adjoint.h", ROOT / "include" / "cfdgpu.h"]))
    out.append((CSRC / "adjoint.cu", BUILD / "adjoint.o", ["--fmad=true", "-DCFD_FAST", "-DCFD_NS=adj"],
                [CSRC / "euler_math.cuh", CSRC / "adjoint.h", CSRC / "adjoint_math.h"]))
    out.append((CSRC / "noalloc.cu", BUILD / "noalloc.o", ["--fmad=false", "-DCFD_NS=api"],
                headers + [CSRC / "sweep_dispatch.h", ROOT / "include" / "cfdgpu.h"]))
    return out


def stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def compile_one(nvcc: str, src: Path, obj: Path, flags: list[str]) -> tuple[Path, int, str]:
    cmd = [nvcc] + common_flags() + flags + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return obj, r.returncode, (r.stdout + r.stderr)


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    nvcc = nvcc_path()
    BUILD.mkdir(exist_ok=True)
    todo = []
    for src, obj, flags, hdrs in units():
        if force or stale(obj, [src] + hdrs + [Path(__file__)]):
            todo.append((src, obj, flags))
    jobs = jobs or max(1, os.cpu_count() or 1)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(compile_one, nvcc, s, o, f) for s, o, f in todo]
            for fu in cf.as_completed(futs):
                obj, rc, log = fu.result()
                if rc != 0:
                    raise RuntimeError(f"nvcc failed for {obj.name}:\n{log}")
                if verbose:
                    print(f"built {obj.name}", flush=True)
    objs = [str(o) for _, o, _, _ in units()]
    if force or todo or not LIB.exists() or any(Path(o).stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(LIB)] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    lib = build(a.jobs, a.force, verbose=True)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
