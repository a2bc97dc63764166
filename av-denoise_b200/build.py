"""Builds libavd_b200.so in-tree with nvcc for sm_100a.

Every `.cu` and `.cpp` under csrc/ is compiled to an object in `_build/` and linked into
`lib/libavd_b200.so` against the static CUDA runtime, so the library loads with no CUDA toolkit
on the library path. Objects are rebuilt only when a source or header is newer.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libavd_b200.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = os.environ.get("NVCC", str(CUDA_HOME / "bin" / "nvcc"))
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-O3,-fvisibility=hidden",
    "-ccbin",
    HOST_CXX,
    f"-I{ROOT / 'include'}",
    f"-I{CSRC}",
]


# Per-file flags. The NL4D collaborative filter rounds every multiply and add on its own, as its CPU
# restatement does (built with -ffp-contract=off), so its member choices and threshold decisions
# agree bit for bit; -fmad=false keeps nvcc from fusing any of them. The noise estimate does the same
# for its reading and fold words, the truemotion stage for its costs and confidences, the exact
# NLMeans finish for its distances, weights and sums, the colour grain gains for their fit, and the
# camera model for its fit and composition.
PER_FILE = {"collab.cu": ["-fmad=false"], "noise_estimate.cu": ["-fmad=false"], "truemotion.cu": ["-fmad=false"],
            "nlm_exact.cu": ["-fmad=false"], "colour.cu": ["-fmad=false"], "camera.cu": ["-fmad=false"]}


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))


def _local_includes(src: Path, seen: set[Path] | None = None) -> set[Path]:
    """The in-tree headers `src` includes, followed recursively (quoted includes only)."""
    seen = set() if seen is None else seen
    for line in src.read_text().splitlines():
        line = line.strip()
        if not line.startswith("#include \""):
            continue
        name = line.split('"')[1]
        for base in (src.parent, CSRC, ROOT / "include"):
            hdr = base / name
            if hdr.exists():
                if hdr not in seen:
                    seen.add(hdr)
                    _local_includes(hdr, seen)
                break
    return seen


def _needs(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = _local_includes(src) & set(headers)
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in deps)


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    cmd = [NVCC, *ARCH, *COMMON, *PER_FILE.get(src.name, []), *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [HOST_CXX, "-std=c++17", "-O3", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
               f"-I{ROOT / 'include'}", f"-I{CSRC}", f"-I{CUDA_HOME / 'include'}", "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles (incrementally) and links the library; returns its path."""
    extra = list(extra or [])
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    srcs = _sources()
    headers = _headers()
    todo = [s for s in srcs if _needs(BUILD / (s.name + ".o"), s, headers)]
    if todo:
        with ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, extra), todo))
    objs = [BUILD / (s.name + ".o") for s in srcs]
    if todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-ccbin", HOST_CXX, "-o", str(LIB), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
