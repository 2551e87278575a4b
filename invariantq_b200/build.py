"""Build libinvariantq.so in-tree with nvcc for sm_100a.

    python -m invariantq_b200.build            # incremental
    python -m invariantq_b200.build --force    # rebuild everything

Objects go to invariantq_b200/_build/, the shared library to
invariantq_b200/libinvariantq.so (the name the reference's ctypes loader looks
for, invariantq/core/binding.py:29).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libinvariantq.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", *ARCH]
SOURCES = ["iq_tile_r3.cu", "iq_tile_r4.cu", "iq_tile_r5.cu", "iq_kernels.cu", "iq_runtime.cu", "iq_sched.cpp", "iq_noalloc.cu",
           "iq_adjoint.cu", "iq_c64.cu", "iq_entropy.cu", "iq_resident.cu", "iq_sampling.cu",
           "iq_selftest.cu", "iq_jit.cpp", "iq_jitgen.cpp"]
HEADERS = ["iq_kernels.h", "iq_plan.h", "iq_pipe.cuh", "iq_tile.cuh", "iq_c64.h", "iq_jit.h", "iq_resident.h"]
# headers the run-time compiled pass kernels include, embedded into the library
JIT_HEADERS = ["iq_plan.h", "iq_pipe.cuh"]
JIT_INC = CSRC / "iq_jit_headers.inc"


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest_dep() -> float:
    deps = [CSRC / h for h in HEADERS] + [JIT_INC, INCLUDE / "invariantq_b200.h", Path(__file__)]
    return max(p.stat().st_mtime for p in deps if p.exists())


def _compile(src: str, force: bool, dep_time: float) -> tuple[str, str]:
    s = CSRC / src
    o = BUILD / (src + ".o")
    if not force and o.exists() and o.stat().st_mtime >= max(s.stat().st_mtime, dep_time):
        return src, ""
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "c++", "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-c", str(s), "-o", str(o)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return src, r.stderr


def _write_jit_headers() -> None:
    """iq_jit_headers.inc: the JIT headers as raw string literals (rewritten
    only when their text changes, so unchanged builds stay incremental)."""
    names, texts = [], []
    for h in JIT_HEADERS:
        t = (CSRC / h).read_text()
        if ")IQJIT\"" in t:
            raise RuntimeError(f"{h} contains the raw-string delimiter")
        names.append(f'"{h}"')
        texts.append(f'R"IQJIT({t})IQJIT"')
    body = ("// generated by invariantq_b200/build.py from " + ", ".join(JIT_HEADERS) + "\n"
            "static const char* const kJitHeaderNames[] = {" + ", ".join(names) + "};\n"
            "static const char* const kJitHeaderSources[] = {\n" + ",\n".join(texts) + "};\n")
    if not JIT_INC.exists() or JIT_INC.read_text() != body:
        JIT_INC.write_text(body)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    _write_jit_headers()
    dep_time = _newest_dep()
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, dep_time), SOURCES))
    if verbose:
        for src, log in results:
            if log:
                print(f"--- {src}\n{log}", file=sys.stderr)
    objs = [BUILD / (s + ".o") for s in SOURCES]
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-cudart", "static", "-ldl", "-lpthread",
               "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
