"""Build libsparsep_b200.so in-tree with nvcc for sm_100a.

Sources: csrc/kernels.cu, csrc/csr_pipe.cu and csrc/csr_stripes.cu (compiled
once per element type, in parallel), csrc/batch_kernels.cu (once per batched type), the other
csrc/*.cu and csrc/*.cpp.  Objects go to sparsep_b200/_build/.
"""
from __future__ import annotations

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
LIB = PKG / "libsparsep_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              f"-I{ROOT / 'include'}", f"-I{CSRC}"]
KERNEL_TYPES = {"i8": "int8_t", "i16": "int16_t", "i32": "int32_t", "i64": "int64_t",
                "f32": "float", "f64": "double"}
BATCH_TYPES = ("f32", "i32")


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(p).exists():
        raise RuntimeError("nvcc not found")
    return p


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")) + list(CSRC.glob("*.cuh"))
                  + list(CSRC.glob("*.hpp")) + [ROOT / "include" / "sparsep.h"])


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    """checked=True builds libsparsep_b200_check.so with -DSPARSEP_CHECK: every
    kernel access is bounds-checked and a failed check is reported as a
    status code instead of touching memory (for diagnosing kernels)."""
    lib_path = LIB.with_name("libsparsep_b200_check.so") if checked else LIB
    bdir = BUILD / ("check" if checked else "release")
    bdir.mkdir(parents=True, exist_ok=True)
    deps = _sources()
    if not force and not _stale(lib_path, deps):
        return lib_path
    flags = NVCC_FLAGS + (["-DSPARSEP_CHECK"] if checked else [])
    jobs = []
    objs = []
    per_type = ("kernels.cu", "csr_pipe.cu", "csr_stripes.cu", "batch_kernels.cu")
    for tag, ctype in KERNEL_TYPES.items():
        for name in per_type[:3]:
            o = bdir / f"{Path(name).stem}_{tag}.o"
            objs.append(o)
            jobs.append([nvcc(), *ARCH, *flags, f"-DSPARSEP_KT={ctype}", "-c", str(CSRC / name), "-o", str(o)])
    for tag in BATCH_TYPES:  # the batched path: FP32 and INT32
        o = bdir / f"batch_kernels_{tag}.o"
        objs.append(o)
        jobs.append([nvcc(), *ARCH, *flags, f"-DSPARSEP_BT={KERNEL_TYPES[tag]}", "-c",
                     str(CSRC / "batch_kernels.cu"), "-o", str(o)])
    for src in sorted(CSRC.glob("*.cu")):
        if src.name in per_type:
            continue
        o = bdir / (src.stem + ".o")
        objs.append(o)
        jobs.append([nvcc(), *ARCH, *flags, "-c", str(src), "-o", str(o)])
    for src in sorted(CSRC.glob("*.cpp")):
        o = bdir / (src.stem + ".o")
        objs.append(o)
        jobs.append([nvcc(), *ARCH, *flags, "-x", "cu", "-c", str(src), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        list(ex.map(_run, jobs))
    tmp = lib_path.with_suffix(".so.tmp")
    _run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
    os.replace(tmp, lib_path)
    if verbose:
        print(f"built {lib_path}")
    return lib_path


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv)
