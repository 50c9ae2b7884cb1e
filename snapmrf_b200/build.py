"""In-tree build of libsnapmrf.so (the C-ABI library) for sm_100a.

Objects go to snapmrf_b200/_build/, the shared library next to this file so
that it travels with the source tree.  Only out-of-date objects are rebuilt.
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
LIB = PKG / "libsnapmrf.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]
SOURCES = ["host.cpp", "ra.cpp", "epg.cu", "match.cu", "match_noalloc.cu", "match_tc.cu", "epg_grad.cu", "epg_ssfp_grad.cu", "refine_start.cu", "svd.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: Path) -> list[Path]:
    deps = [src] + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    return [d for d in deps if d.exists()]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: str, verbose: bool, extra: list[str]) -> Path:
    s = CSRC / src
    obj = BUILD / (s.stem + ".o")
    if _stale(obj, _deps(s)):
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", str(s), "-o", str(obj)]
        if s.suffix == ".cpp":
            cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + extra + ["-c", str(s), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
    return obj


COMPAT_LIB = PKG / "libsnapmrf_compat.so"
# the benchmark's FP32 FMA throughput probe (not part of the product library)
PROBE_LIB = PKG / "libsnapmrf_probe.so"
CLI = PKG / "mrf"
RPATH = ["-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]


def _link(target: Path, objs: list[Path], extra: list[str]) -> None:
    if not _stale(target, objs + ([LIB] if target != LIB else [])):
        return
    tmp = target.with_name(target.name + ".tmp")
    cmd = [nvcc()] + ARCH + extra + ["-o", str(tmp)] + [str(o) for o in objs]
    if target != LIB:
        cmd += [f"-L{PKG}", "-lsnapmrf"] + RPATH
    cmd += ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link of {target.name} failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, target)


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles every CUDA/C++ source, links libsnapmrf.so, the functions.h
    compatibility library libsnapmrf_compat.so and the mrf CLI; returns the
    path of libsnapmrf.so."""
    BUILD.mkdir(exist_ok=True)
    extra = list(extra or [])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra),
                           SOURCES + ["compat.cpp", "mrf_cli.cpp", "fp32_probe.cu"]))
    core, compat_o, cli_o, probe_o = objs[:len(SOURCES)], objs[-3], objs[-2], objs[-1]
    _link(LIB, core, ["-shared"])
    _link(COMPAT_LIB, [compat_o], ["-shared"])
    _link(CLI, [cli_o], [])
    if _stale(PROBE_LIB, [probe_o]):
        tmp = PROBE_LIB.with_name(PROBE_LIB.name + ".tmp")
        r = subprocess.run([nvcc()] + ARCH + ["-shared", "-o", str(tmp), str(probe_o), "-lcudart"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of {PROBE_LIB.name} failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, PROBE_LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
